// eig_batched.cu -- batched FP64 symmetric eigensolver kernels (one CTA per block).
// See eig_batched.cuh for the role of each stage and the reference routines replaced.
#include <algorithm>
#include <cfloat>
#include <cmath>

#include "common.cuh"
#include "eig_batched.cuh"
#include "tridiag_dev.cuh"

namespace dvr3d {

namespace {

constexpr int kTriMaxThreads = 1024;  // one row per thread -> n <= 1024

// ------------------------------------------------------------------ tridiagonalisation
// Lower Householder reduction as dsytd2('L'): for k = 0..n-3 the reflector
// H_k = I - tau_k v v^T, v = (0..0, 1, v_{k+2..n-1}), annihilates A[k+2:, k].
// The rank-2 update of step k-1 is applied lazily: to column k first (so the reflector
// of step k can be formed), then fused with the symmetric product A22 v_k of step k, so
// the trailing block is read and written once per step.
__global__ void __launch_bounds__(kTriMaxThreads) tridiag_kernel(BatchDesc bd, double *A, double *dg,
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
        // (3) fused: apply pending update to A22 and accumulate s = A22 v. One row per thread,
        // or per pair of adjacent threads (the two take alternate columns) when the block has
        // threads to spare: twice the loads in flight per row. Four columns per iteration.
        const int R = (blockDim.x >= 2u * (unsigned)n) ? 2 : 1;
        const int i = k + 1 + tid / R, h = tid % R;
        const bool act = i < n;
        const double vpi = (pending && act) ? vp[i] : 0.0, wpi = (pending && act) ? wp[i] : 0.0;
        double s_acc = 0.0;
        if (act && (tk != 0.0 || pending)) {
            const size_t sn = (size_t)R * n;  // stride between this thread's columns
            int j = k + 1 + h;
            for (; j + 3 * R < n; j += 4 * R) {
                double *c0 = a + (size_t)j * n + i;
                double x0 = c0[0], x1 = c0[sn], x2 = c0[2 * sn], x3 = c0[3 * sn];
                if (pending) {
                    x0 -= vpi * wp[j] + wpi * vp[j];
                    x1 -= vpi * wp[j + R] + wpi * vp[j + R];
                    x2 -= vpi * wp[j + 2 * R] + wpi * vp[j + 2 * R];
                    x3 -= vpi * wp[j + 3 * R] + wpi * vp[j + 3 * R];
                    c0[0] = x0;
                    c0[sn] = x1;
                    c0[2 * sn] = x2;
                    c0[3 * sn] = x3;
                }
                s_acc += (x0 * v[j] + x1 * v[j + R]) + (x2 * v[j + 2 * R] + x3 * v[j + 3 * R]);
            }
            for (; j < n; j += R) {
                double *cj = a + (size_t)j * n + i;
                double x = *cj;
                if (pending) {
                    x -= vpi * wp[j] + wpi * vp[j];
                    *cj = x;
                }
                s_acc += x * v[j];
            }
        }
        if (R == 2) s_acc += __shfl_xor_sync(0xffffffffu, s_acc, 1);  // partner thread, same warp
        // p = tau s ; w = p - (tau/2)(p.v) v
        double pv = (act && h == 0) ? tk * s_acc * v[i] : 0.0;
        pv = block_sum(pv, red);
        const double alpha2 = -0.5 * tk * pv;
        __syncthreads();
        for (int q = tid; q < n; q += blockDim.x) {
            vp[q] = v[q];
            wp[q] = 0.0;
        }
        __syncthreads();
        if (act && h == 0) wp[i] = tk * s_acc + alpha2 * v[i];
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
            invit_cluster(d, e, n, w, cstart[c], cstart[c + 1], s_onenrm, fac, T, tid, X, m, err);
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

// ------------------------------------------------------------------ eigenvectors, fast form
// Same method as eigvecs_kernel (dstein-style inverse iteration, Gram-Schmidt inside clusters
// closer than 1e-6 ||T||, back-transformation by the block's reflectors), organised for speed:
//   * one warp per cluster, the LU factors of T - lambda I and the iterate in that warp's
//     slice of shared memory (lane 0 runs the recurrences, the warp the vector operations);
//   * the back-transformation in panels of 16 reflectors (compact WY, I - V Tm V^T): per
//     panel V and Tm in shared memory, one thread per eigenvector column computing
//     W = V^T z, W2 = Tm W and z -= V W2 in registers.
constexpr int kFastPanel = 16;

// The first vector of eigvecs_fast_kernel that failed its growth test since the last clear:
// {failed, block, eigenvalue index, block order}, for the host's error message.
__device__ int g_invit_fail[4];

__global__ void eigvecs_fast_kernel(BatchDesc bd, const double *A, const double *dg, const double *eo,
                                    const double *tauo, const double *wo, const int *sel, const long long *zoff,
                                    const int *zld, double *Z, int *err) {
    // gridDim.y CTAs share a block: CTA y takes the eigenvalue clusters c = y (mod gridDim.y)
    // and back-transforms their columns
    const int b = blockIdx.x, part = blockIdx.y, nparts = gridDim.y;
    if (b >= bd.nblk) return;
    const int n = bd.n[b];
    const int m = sel[b];
    if (m <= 0) return;
    const double *a = A + bd.aoff[b];
    const double *d = dg + bd.voff[b], *e = eo + bd.voff[b], *tau = tauo + bd.voff[b];
    const double *w = wo + bd.voff[b];
    double *z = Z + zoff[b];
    const int ldz = zld[b];
    extern __shared__ double sm[];
    __shared__ int cstart[1025];
    __shared__ int mycols[1024];  // columns of this CTA's clusters
    __shared__ int s_ncl, s_nmine;
    __shared__ double s_onenrm;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = blockDim.x >> 5;
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
        int nm = 0;
        for (int c = part; c < nc; c += nparts)
            for (int j = cstart[c]; j < cstart[c + 1]; ++j) mycols[nm++] = j;
        s_nmine = nm;
    }
    __syncthreads();
    // ---- inverse iteration, one warp per cluster
    {
        const size_t slice = (size_t)5 * n + (n + 7) / 8;  // doubles per warp
        double *D = sm + warp * slice, *E1 = D + n, *E2 = E1 + n, *Lm = E2 + n, *x = Lm + n;
        unsigned char *P = reinterpret_cast<unsigned char *>(x + n);
        const double onenrm = s_onenrm;
        const double eps = DBL_EPSILON, tiny = eps * onenrm, pertol = 10.0 * eps * onenrm;
        for (int c = part + nparts * warp; c < s_ncl; c += nparts * nwarp) {
            const int j0 = cstart[c], j1 = cstart[c + 1];
            double lamprev = 0.0;
            for (int j = j0; j < j1; ++j) {
                double lam = w[j];
                if (j > j0 && lam - lamprev < pertol) lam = lamprev + pertol;
                lamprev = lam;
                if (lane == 0) {
                    double av = d[0] - lam, bv = (n > 1) ? e[0] : 0.0;
                    for (int i = 0; i < n - 1; ++i) {
                        const double cc = e[i];
                        const double an = d[i + 1] - lam, bn = (i + 2 < n) ? e[i + 1] : 0.0;
                        if (fabs(av) >= fabs(cc)) {
                            if (av == 0.0) av = tiny;
                            const double mlt = cc / av;
                            P[i] = 0;
                            Lm[i] = mlt;
                            D[i] = av;
                            E1[i] = bv;
                            E2[i] = 0.0;
                            av = an - mlt * bv;
                            bv = bn;
                        } else {
                            const double mlt = av / cc;
                            P[i] = 1;
                            Lm[i] = mlt;
                            D[i] = cc;
                            E1[i] = an;
                            E2[i] = bn;
                            av = bv - mlt * an;
                            bv = -mlt * bn;
                        }
                    }
                    if (fabs(av) < tiny) av = (av < 0.0) ? -tiny : tiny;
                    D[n - 1] = av;
                    // no superdiagonals in the last row of U; the back substitution reads them
                    // (times zero), so stale shared memory must not leave a NaN there
                    E1[n - 1] = 0.0;
                    E2[n - 1] = 0.0;
                }
                __syncwarp();
                for (int i = lane; i < n - 1; i += 32)
                    if (fabs(D[i]) < tiny) D[i] = (D[i] < 0.0) ? -tiny : tiny;
                __syncwarp();
                // the solves below multiply by the pivots' reciprocals (one division per pivot
                // here instead of one per pivot and iteration on the sequential path)
                const double dlast = D[n - 1];
                __syncwarp();
                for (int i = lane; i < n; i += 32) D[i] = 1.0 / D[i];
                for (int i = lane; i < n; i += 32) {
                    const unsigned h = hash32((unsigned)(i * 2654435761u) ^ (unsigned)(j * 40503u + 17u));
                    x[i] = ((double)(h & 0xffffff) / 8388608.0) - 1.0;
                }
                __syncwarp();
                const double grow_lim = invit_growth_limit(n);
                int grown = 0;
                for (int it = 0; it < kInvitPasses; ++it) {
                    double s1 = 0.0;
                    for (int i = lane; i < n; i += 32) s1 += fabs(x[i]);
                    s1 = warp_sum(s1);
                    const double sc = (double)n * onenrm * fmax(eps, fabs(dlast)) / fmax(s1, DBL_MIN);
                    for (int i = lane; i < n; i += 32) x[i] *= sc;
                    __syncwarp();
                    if (lane == 0) {
                        for (int i = 0; i < n - 1; ++i) {
                            double yi = x[i], yn = x[i + 1];
                            if (P[i]) {
                                const double tmp = yi;
                                yi = yn;
                                yn = tmp;
                                x[i] = yi;
                            }
                            x[i + 1] = yn - Lm[i] * yi;
                        }
                        double x1 = 0.0, x2 = 0.0;
                        for (int i = n - 1; i >= 0; --i) {
                            const double xi = (x[i] - E1[i] * x1 - E2[i] * x2) * D[i];
                            x[i] = xi;
                            x2 = x1;
                            x1 = xi;
                        }
                    }
                    __syncwarp();
                    for (int jj = j0; jj < j; ++jj) {
                        const double *zc = z + (size_t)jj * ldz;
                        double dot = 0.0;
                        for (int i = lane; i < n; i += 32) dot += x[i] * zc[i];
                        dot = warp_sum(dot);
                        for (int i = lane; i < n; i += 32) x[i] -= dot * zc[i];
                    }
                    double nrm = 0.0, xinf = 0.0;
                    for (int i = lane; i < n; i += 32) {
                        nrm += x[i] * x[i];
                        xinf = fmax(xinf, fabs(x[i]));
                    }
                    nrm = sqrt(warp_sum(nrm));
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) xinf = fmax(xinf, __shfl_xor_sync(0xffffffffu, xinf, o));
                    grown += (xinf >= grow_lim);
                    const double inv = (nrm > 0.0) ? 1.0 / nrm : 0.0;
                    for (int i = lane; i < n; i += 32) x[i] *= inv;
                    __syncwarp();
                }
                if (grown < kInvitGrowPasses && lane == 0 && err) {
                    *err = kDevNoConv;
                    if (atomicCAS(&g_invit_fail[0], 0, 1) == 0) {
                        g_invit_fail[1] = b;
                        g_invit_fail[2] = j;
                        g_invit_fail[3] = n;
                    }
                }
                // sign convention: the first largest component positive
                double big = 0.0;
                int bi = n;
                for (int i = lane; i < n; i += 32)
                    if (fabs(x[i]) > fabs(big)) {
                        big = x[i];
                        bi = i;
                    }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    const double ob = __shfl_xor_sync(0xffffffffu, big, o);
                    const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                    if (fabs(ob) > fabs(big) || (fabs(ob) == fabs(big) && oi < bi)) {
                        big = ob;
                        bi = oi;
                    }
                }
                const double sg = (big < 0.0) ? -1.0 : 1.0;
                double *zc = z + (size_t)j * ldz;
                for (int i = lane; i < n; i += 32) zc[i] = sg * x[i];
                __syncwarp();
            }
        }
    }
    __syncthreads();
    // ---- back-transformation z <- H_0 H_1 ... H_{n-3} z, panels of 16 reflectors
    const int nref = n - 2;
    if (nref <= 0) return;
    double *Vs = sm;                                   // [kFastPanel][n]
    double *Sg = Vs + (size_t)kFastPanel * n;          // [16][16] Gram, then
    double *Tm = Sg + kFastPanel * kFastPanel;         // [16][16] upper triangular factor
    for (int p0 = ((nref - 1) / kFastPanel) * kFastPanel; p0 >= 0; p0 -= kFastPanel) {
        const int nbk = min(kFastPanel, nref - p0);
        for (int q = tid; q < kFastPanel * n; q += blockDim.x) {
            const int c = q / n, i = q % n, top = p0 + c + 1;
            double v = 0.0;
            if (c < nbk && i >= top) v = (i == top) ? 1.0 : a[(size_t)(p0 + c) * n + i];
            Vs[q] = v;
        }
        __syncthreads();
        for (int q = tid; q < kFastPanel * kFastPanel; q += blockDim.x) {
            const int c1 = q / kFastPanel, c2 = q % kFastPanel;
            double s = 0.0;
            if (c1 < nbk && c2 < nbk)
                for (int i = p0 + 1; i < n; ++i) s += Vs[c1 * n + i] * Vs[c2 * n + i];
            Sg[q] = s;
        }
        __syncthreads();
        if (tid < kFastPanel) {  // dlarft (forward, columnwise), one thread per row of Tm
            const int r = tid;
            for (int c = 0; c < kFastPanel; ++c) Tm[r * kFastPanel + c] = 0.0;
        }
        __syncthreads();
        for (int i = 0; i < nbk; ++i) {
            if (tid < kFastPanel) {
                const int r = tid;
                const double ti = tau[p0 + i];
                if (r < i) {
                    double s = 0.0;
                    for (int c = r; c < i; ++c) s += Tm[r * kFastPanel + c] * Sg[c * kFastPanel + i];
                    Tm[r * kFastPanel + i] = -ti * s;
                } else if (r == i) {
                    Tm[i * kFastPanel + i] = ti;
                }
            }
            __syncthreads();
        }
        for (int q = tid; q < s_nmine; q += blockDim.x) {
            double *zc = z + (size_t)mycols[q] * ldz;
            // the column is walked four rows at a time so that four loads are in flight
            double wv[kFastPanel];
#pragma unroll
            for (int c = 0; c < kFastPanel; ++c) wv[c] = 0.0;
            int i = p0 + 1;
            for (; i + 3 < n; i += 4) {
                const double z0 = zc[i], z1 = zc[i + 1], z2 = zc[i + 2], z3 = zc[i + 3];
#pragma unroll
                for (int c = 0; c < kFastPanel; ++c) {
                    const double *vc = Vs + c * n + i;
                    wv[c] += (vc[0] * z0 + vc[1] * z1) + (vc[2] * z2 + vc[3] * z3);
                }
            }
            for (; i < n; ++i) {
                const double zi = zc[i];
#pragma unroll
                for (int c = 0; c < kFastPanel; ++c) wv[c] += Vs[c * n + i] * zi;
            }
            double w2[kFastPanel];
#pragma unroll
            for (int r = 0; r < kFastPanel; ++r) {
                double s = 0.0;
#pragma unroll
                for (int c = 0; c < kFastPanel; ++c) s += Tm[r * kFastPanel + c] * wv[c];
                w2[r] = s;
            }
            i = p0 + 1;
            for (; i + 3 < n; i += 4) {
                const double z0 = zc[i], z1 = zc[i + 1], z2 = zc[i + 2], z3 = zc[i + 3];
                double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
#pragma unroll
                for (int c = 0; c < kFastPanel; ++c) {
                    const double *vc = Vs + c * n + i;
                    s0 += vc[0] * w2[c];
                    s1 += vc[1] * w2[c];
                    s2 += vc[2] * w2[c];
                    s3 += vc[3] * w2[c];
                }
                zc[i] = z0 - s0;
                zc[i + 1] = z1 - s1;
                zc[i + 2] = z2 - s2;
                zc[i + 3] = z3 - s3;
            }
            for (; i < n; ++i) {
                double s = 0.0;
#pragma unroll
                for (int c = 0; c < kFastPanel; ++c) s += Vs[c * n + i] * w2[c];
                zc[i] -= s;
            }
        }
        __syncthreads();
    }
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
    // two threads per row while 2 nmax fits in one block (see the fused loop)
    const int rows_thr = (2 * nmax <= kTriMaxThreads) ? 2 * nmax : nmax;
    const int threads = std::min(kTriMaxThreads, std::max(64, (rows_thr + 31) / 32 * 32));
    tridiag_kernel<<<bd.nblk, threads, smem, st>>>(bd, A, d, e, tau);
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

size_t eigvecs_fast_smem(int nmax, int nwarp) {
    const size_t inv = (size_t)nwarp * (5 * (size_t)nmax + (nmax + 7) / 8) * sizeof(double);
    const size_t bt = ((size_t)kFastPanel * nmax + 2 * kFastPanel * kFastPanel) * sizeof(double);
    return std::max(inv, bt);
}

void launch_eigvecs_batched_fast(const BatchDesc &bd, const double *A, const double *d, const double *e,
                                 const double *tau, const double *w, const int *sel, const long long *zoff,
                                 const int *zld, double *Z, int nmax, int *err, cudaStream_t st) {
    if (bd.nblk <= 0) return;
    const size_t cap = 200 * 1024;
    int nwarp = 8;
    while (nwarp > 1 && eigvecs_fast_smem(nmax, nwarp) > cap) --nwarp;
    const size_t smem = eigvecs_fast_smem(nmax, nwarp);
    // fewer blocks than SMs: two CTAs per block (their clusters split between them)
    int dev = 0, nsm = 0;
    cudaGetDevice(&dev);
    // the shared-memory limit is a per-device attribute of the kernel
    static bool attr[kMaxAttrDevices] = {};
    if (dev < 0 || dev >= kMaxAttrDevices || !attr[dev]) {
        cudaFuncSetAttribute(eigvecs_fast_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cap);
        if (dev >= 0 && dev < kMaxAttrDevices) attr[dev] = true;
    }
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const int parts = (bd.nblk < nsm) ? 2 : 1;
    DVR3D_COUNT_LAUNCH(1);
    eigvecs_fast_kernel<<<dim3(bd.nblk, parts), 32 * nwarp, smem, st>>>(bd, A, d, e, tau, w, sel, zoff, zld, Z, err);
}

void invit_fail_clear(cudaStream_t st) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_invit_fail) == cudaSuccess) cudaMemsetAsync(p, 0, sizeof(int) * 4, st);
}

void invit_fail_info(cudaStream_t st, int out[4]) {
    void *p = nullptr;
    out[0] = out[1] = out[2] = out[3] = 0;
    if (cudaGetSymbolAddress(&p, g_invit_fail) == cudaSuccess) {
        cudaMemcpyAsync(out, p, sizeof(int) * 4, cudaMemcpyDeviceToHost, st);
        cudaStreamSynchronize(st);
    }
}

}  // namespace dvr3d
