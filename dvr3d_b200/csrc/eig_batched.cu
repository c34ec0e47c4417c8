// eig_batched.cu -- batched FP64 symmetric eigensolver kernels (one CTA per block).
// See eig_batched.cuh for the role of each stage and the reference routines replaced.
#include <cfloat>
#include <cmath>

#include "common.cuh"
#include "eig_batched.cuh"
#include "tridiag_dev.cuh"

namespace dvr3d {

namespace {

constexpr int kTriThreads = 256;
constexpr int kTriRows = 4;  // rows per thread -> n <= 1024

// ------------------------------------------------------------------ tridiagonalisation
// Lower Householder reduction as dsytd2('L'): for k = 0..n-3 the reflector
// H_k = I - tau_k v v^T, v = (0..0, 1, v_{k+2..n-1}), annihilates A[k+2:, k].
// The rank-2 update of step k-1 is applied lazily: to column k first (so the reflector
// of step k can be formed), then fused with the symmetric product A22 v_k of step k, so
// the trailing block is read and written once per step.
__global__ void __launch_bounds__(kTriThreads) tridiag_kernel(BatchDesc bd, double *A, double *dg,
                                                               double *eo, double *tauo) {
    const int b = blockIdx.x;
    if (b >= bd.nblk) return;
    const int n = bd.n[b];
    double *a = A + bd.aoff[b];
    double *d = dg + bd.voff[b], *e = eo + bd.voff[b], *tau = tauo + bd.voff[b];
    extern __shared__ double sm[];
    double *vp = sm, *wp = sm + n, *v = sm + 2 * n;  // pending (v, w) and current v
    __shared__ double red[32];
    __shared__ double s_beta, s_tau, s_scal;
    const int tid = threadIdx.x;
    if (n == 1) {
        if (tid == 0) {
            d[0] = a[0];
            e[0] = 0.0;
            tau[0] = 0.0;
        }
        return;
    }
    bool pending = false;
    for (int k = 0; k + 2 < n; ++k) {
        // (1) finish column k: A[i,k] -= vp_i wp_k + wp_i vp_k, i >= k
        if (pending) {
            const double vk = vp[k], wk = wp[k];
            for (int i = k + tid; i < n; i += blockDim.x) a[(size_t)k * n + i] -= vp[i] * wk + wp[i] * vk;
        }
        __syncthreads();
        // (2) Householder vector from x = A[k+1:, k]
        double ss = 0.0;
        for (int i = k + 2 + tid; i < n; i += blockDim.x) {
            const double x = a[(size_t)k * n + i];
            ss += x * x;
        }
        ss = block_sum(ss, red);
        if (tid == 0) {
            const double alpha = a[(size_t)k * n + k + 1];
            d[k] = a[(size_t)k * n + k];
            if (ss == 0.0) {
                s_tau = 0.0;
                s_beta = alpha;
                s_scal = 0.0;
            } else {
                const double beta = -copysign(sqrt(alpha * alpha + ss), alpha);
                s_tau = (beta - alpha) / beta;
                s_beta = beta;
                s_scal = 1.0 / (alpha - beta);
            }
            e[k] = s_beta;
            tau[k] = s_tau;
        }
        __syncthreads();
        const double tk = s_tau, scal = s_scal;
        for (int i = tid; i < n; i += blockDim.x) {
            double vi = 0.0;
            if (i == k + 1) vi = 1.0;
            else if (i > k + 1) {
                vi = a[(size_t)k * n + i] * scal;
                a[(size_t)k * n + i] = vi;  // reflector kept below the subdiagonal
            }
            v[i] = vi;
        }
        __syncthreads();
        // (3) fused: apply pending update to A22 and accumulate s = A22 v
        double s_acc[kTriRows];
        double vpi[kTriRows], wpi[kTriRows];
#pragma unroll
        for (int r = 0; r < kTriRows; ++r) {
            s_acc[r] = 0.0;
            const int i = k + 1 + tid + r * blockDim.x;
            vpi[r] = (pending && i < n) ? vp[i] : 0.0;
            wpi[r] = (pending && i < n) ? wp[i] : 0.0;
        }
        if (tk != 0.0 || pending) {
            for (int j = k + 1; j < n; ++j) {
                double *col = a + (size_t)j * n;
                const double vj = v[j];
                const double vpj = pending ? vp[j] : 0.0, wpj = pending ? wp[j] : 0.0;
#pragma unroll
                for (int r = 0; r < kTriRows; ++r) {
                    const int i = k + 1 + tid + r * blockDim.x;
                    if (i < n) {
                        double x = col[i];
                        if (pending) {
                            x -= vpi[r] * wpj + wpi[r] * vpj;
                            col[i] = x;
                        }
                        s_acc[r] += x * vj;
                    }
                }
            }
        }
        // p = tau s ; w = p - (tau/2)(p.v) v
        double pv = 0.0;
#pragma unroll
        for (int r = 0; r < kTriRows; ++r) {
            const int i = k + 1 + tid + r * blockDim.x;
            if (i < n) pv += tk * s_acc[r] * v[i];
        }
        pv = block_sum(pv, red);
        const double alpha2 = -0.5 * tk * pv;
        __syncthreads();
        for (int i = tid; i < n; i += blockDim.x) {
            vp[i] = v[i];
            wp[i] = 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < kTriRows; ++r) {
            const int i = k + 1 + tid + r * blockDim.x;
            if (i < n) wp[i] = tk * s_acc[r] + alpha2 * v[i];
        }
        pending = (tk != 0.0);
        __syncthreads();
    }
    // trailing 2x2 block
    if (tid == 0) {
        double a00 = a[(size_t)(n - 2) * n + (n - 2)];
        double a10 = a[(size_t)(n - 2) * n + (n - 1)];
        double a11 = a[(size_t)(n - 1) * n + (n - 1)];
        if (pending) {
            a00 -= 2.0 * vp[n - 2] * wp[n - 2];
            a10 -= vp[n - 1] * wp[n - 2] + wp[n - 1] * vp[n - 2];
            a11 -= 2.0 * vp[n - 1] * wp[n - 1];
        }
        d[n - 2] = a00;
        d[n - 1] = a11;
        e[n - 2] = a10;
        e[n - 1] = 0.0;
        tau[n - 2] = 0.0;
        tau[n - 1] = 0.0;
    }
}

constexpr int kEvThreads = 256;

__global__ void __launch_bounds__(kEvThreads) eigvals_kernel(BatchDesc bd, const double *dg,
                                                              const double *eo, double *wo,
                                                              int *cnt, int mode, double cut) {
    const int b = blockIdx.x;
    if (b >= bd.nblk) return;
    const int n = bd.n[b];
    const double *d = dg + bd.voff[b], *e = eo + bd.voff[b];
    double *w = wo + bd.voff[b];
    extern __shared__ double sm[];
    double *sd = sm, *e2 = sm + n;
    __shared__ double red[32];
    __shared__ int s_count;
    __shared__ double s_lo, s_hi, s_piv;
    const int tid = threadIdx.x;
    double lo = DBL_MAX, hi = -DBL_MAX, emx = 0.0;
    for (int i = tid; i < n; i += blockDim.x) {
        const double di = d[i];
        const double em = (i > 0) ? fabs(e[i - 1]) : 0.0, ep = (i < n - 1) ? fabs(e[i]) : 0.0;
        sd[i] = di;
        if (i < n - 1) e2[i] = e[i] * e[i];
        lo = fmin(lo, di - em - ep);
        hi = fmax(hi, di + em + ep);
        emx = fmax(emx, (i < n - 1) ? e[i] * e[i] : 0.0);
    }
    // block min / max via the sum helper on negated / shifted values is awkward: use shared
    __shared__ double s_min[kEvThreads], s_max[kEvThreads], s_e[kEvThreads];
    s_min[tid] = lo;
    s_max[tid] = hi;
    s_e[tid] = emx;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (tid < s) {
            s_min[tid] = fmin(s_min[tid], s_min[tid + s]);
            s_max[tid] = fmax(s_max[tid], s_max[tid + s]);
            s_e[tid] = fmax(s_e[tid], s_e[tid + s]);
        }
        __syncthreads();
    }
    if (tid == 0) {
        const double tnorm = fmax(fabs(s_min[0]), fabs(s_max[0]));
        s_piv = DBL_MIN * fmax(1.0, s_e[0]);
        s_lo = s_min[0] - 2.0 * DBL_EPSILON * tnorm * n - 2.0 * s_piv;
        s_hi = s_max[0] + 2.0 * DBL_EPSILON * tnorm * n + 2.0 * s_piv;
    }
    __syncthreads();
    (void)red;
    int m = n;
    if (mode != 0) {
        if (tid == 0) {
            double x = cut;
            if (mode == 2) x = nextafter(cut, DBL_MAX);  // count of eigenvalues <= cut
            s_count = (x <= s_lo) ? 0 : (x >= s_hi ? n : sturm_count(sd, e2, n, x, s_piv));
        }
        __syncthreads();
        m = s_count;
    }
    if (tid == 0) cnt[b] = m;
    for (int j = tid; j < m; j += blockDim.x) w[j] = bisect_one(sd, e2, n, j, s_lo, s_hi, s_piv);
}

// ------------------------------------------------------------------ inverse iteration
constexpr int kVecThreads = 128;

__global__ void __launch_bounds__(kVecThreads) eigvecs_kernel(BatchDesc bd, const double *A,
                                                               const double *dg, const double *eo,
                                                               const double *tauo, const double *wo,
                                                               const int *sel, const long long *zoff,
                                                               const int *zld, double *Z, double *work,
                                                               const long long *workoff, int *err) {
    const int b = blockIdx.x;
    if (b >= bd.nblk) return;
    const int n = bd.n[b];
    const int m = sel[b];
    if (m <= 0) return;
    const double *a = A + bd.aoff[b];
    const double *d = dg + bd.voff[b], *e = eo + bd.voff[b], *tau = tauo + bd.voff[b];
    const double *w = wo + bd.voff[b];
    double *z = Z + zoff[b];
    const int ldz = zld[b];
    double *wk = work + workoff[b];
    extern __shared__ double sm[];
    int *cstart = reinterpret_cast<int *>(sm);  // cluster starts (m+1 ints)
    __shared__ int s_ncl;
    __shared__ double s_onenrm;
    const int tid = threadIdx.x;
    // clusters: consecutive eigenvalues closer than 1e-6 ||T||_1 are orthogonalised
    if (tid == 0) {
        double on = 0.0;
        for (int i = 0; i < n; ++i) {
            const double r = fabs(d[i]) + (i > 0 ? fabs(e[i - 1]) : 0.0) + (i < n - 1 ? fabs(e[i]) : 0.0);
            on = fmax(on, r);
        }
        s_onenrm = fmax(on, DBL_MIN);
        const double ortol = 1.0e-6 * s_onenrm;
        int nc = 0;
        cstart[nc++] = 0;
        for (int j = 1; j < m; ++j)
            if (w[j] - w[j - 1] > ortol) cstart[nc++] = j;
        cstart[nc] = m;
        s_ncl = nc;
    }
    __syncthreads();
    const int ncl = s_ncl;
    const int T = min((int)blockDim.x, m);   // thread slots holding LU factors
    double *fac = wk;                        // 5 * n * T
    double *X = wk + (size_t)5 * n * T;      // n * m, interleaved by eigenvalue
    if (tid < T)
        for (int c = tid; c < ncl; c += T)
            invit_cluster(d, e, n, w, cstart[c], cstart[c + 1], s_onenrm, fac, T, tid, X, m);
    __syncthreads();
    const int TT = blockDim.x;
    // copy to Z (column per eigenvalue) -- coalesced over rows
    for (int idx = tid; idx < n * m; idx += TT) {
        const int jcol = idx / n, i = idx - jcol * n;
        z[(size_t)jcol * ldz + i] = X[(size_t)i * m + jcol];
    }
    __syncthreads();
    // back-transform: z <- H_0 H_1 ... H_{n-3} z  (apply H_{n-3} first)
    double *vs = sm;  // reuse shared memory for the reflector
    const int lane = tid & 31, wid = tid >> 5, nw = TT >> 5;
    for (int k = n - 3; k >= 0; --k) {
        const double tk = tau[k];
        __syncthreads();
        if (tk == 0.0) continue;
        for (int i = k + 1 + tid; i < n; i += TT) vs[i] = (i == k + 1) ? 1.0 : a[(size_t)k * n + i];
        __syncthreads();
        for (int jcol = wid; jcol < m; jcol += nw) {
            double *zc = z + (size_t)jcol * ldz;
            double s = 0.0;
            for (int i = k + 1 + lane; i < n; i += 32) s += vs[i] * zc[i];
            s = warp_sum(s) * tk;
            for (int i = k + 1 + lane; i < n; i += 32) zc[i] -= s * vs[i];
        }
    }
    (void)err;
}

__global__ void symmetrize_lower_kernel(BatchDesc bd, double *A) {
    const int b = blockIdx.y;
    const int n = bd.n[b];
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)n * n) return;
    const int i = (int)(idx % n), j = (int)(idx / n);
    if (j > i) A[bd.aoff[b] + idx] = A[bd.aoff[b] + (long long)i * n + j];
}

}  // namespace

void launch_symmetrize_lower(const BatchDesc &bd, double *A, int nmax, cudaStream_t st) {
    dim3 grid((unsigned)(((long long)nmax * nmax + 255) / 256), bd.nblk);
    DVR3D_COUNT_LAUNCH(1);
    symmetrize_lower_kernel<<<grid, 256, 0, st>>>(bd, A);
}

void launch_tridiag_batched(const BatchDesc &bd, double *A, double *d, double *e, double *tau,
                            int nmax, cudaStream_t st) {
    if (bd.nblk <= 0) return;
    const size_t smem = (size_t)3 * nmax * sizeof(double);
    DVR3D_COUNT_LAUNCH(1);
    tridiag_kernel<<<bd.nblk, kTriThreads, smem, st>>>(bd, A, d, e, tau);
}

void launch_eigvals_batched(const BatchDesc &bd, const double *d, const double *e, double *w,
                            int *cnt, int mode, double cut, cudaStream_t st) {
    if (bd.nblk <= 0) return;
    int nmax = 0;
    (void)nmax;
    // dynamic shared memory: d and e^2 of the largest block (caller guarantees <= 1024)
    DVR3D_COUNT_LAUNCH(1);
    eigvals_kernel<<<bd.nblk, kEvThreads, 2 * 1024 * sizeof(double), st>>>(bd, d, e, w, cnt, mode, cut);
}

void launch_eigvecs_batched(const BatchDesc &bd, const double *A, const double *d,
                            const double *e, const double *tau, const double *w,
                            const int *sel, const long long *zoff, const int *zld, double *Z,
                            double *work, const long long *workoff, int nmax, int *err,
                            cudaStream_t st) {
    if (bd.nblk <= 0) return;
    size_t smem = (size_t)nmax * sizeof(double);
    const size_t smem_cl = (size_t)(nmax + 2) * sizeof(int);
    if (smem_cl > smem) smem = smem_cl;
    DVR3D_COUNT_LAUNCH(1);
    eigvecs_kernel<<<bd.nblk, kVecThreads, smem, st>>>(bd, A, d, e, tau, w, sel, zoff, zld, Z, work,
                                                       workoff, err);
}

}  // namespace dvr3d
