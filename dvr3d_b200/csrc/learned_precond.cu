// learned_precond.cu -- channel-block preconditioner kernels and the forward / backward / Adam
// kernels of its learned spectral correction (model: learned_precond.cuh).
//
// Parameter layout (doubles): W1[16][4] @0, b1[16] @64, W2[16][16] @80, b2[16] @336,
// w3[16] @352, b3 @368.
// Channel kernels: one CTA per (channel, 16 columns); Q_c and the gathered rows of the
// channel sit in shared memory, the two small products Q^T r and Q z are done there.
// MLP gradient: chunks of 128 (mode, column) items per CTA; one thread per item computes the
// activations and back-propagated deltas into shared memory, then one thread per parameter
// sums its gradient over the chunk; per-CTA partials are reduced in a second kernel
// (deterministic order).
#include <algorithm>
#include <cmath>

#include "common.cuh"
#include "learned_precond.cuh"

namespace dvr3d {

namespace {

constexpr int F = kLpFeat, Hd = kLpHidden;
constexpr int oW1 = 0, oB1 = Hd * F, oW2 = oB1 + Hd, oB2 = oW2 + Hd * Hd, oW3 = oB2 + Hd, oB3 = oW3 + Hd;
static_assert(oB3 + 1 == kLpParams, "parameter layout");
constexpr int kCols = 16;    // columns per channel CTA
constexpr int kChunk = 128;  // items per MLP-gradient chunk
constexpr int kItem = F + Hd + Hd + 1 + Hd + Hd;  // phi, z1, z2, delta, d2, d1
constexpr int kGradGrid = 296;

__device__ __forceinline__ double safe_den(double d) {
    const double eps = 1.0e-4;
    return fabs(d) < eps ? (d < 0.0 ? -eps : eps) : d;
}

__device__ __forceinline__ void features(const LpModes &m, int i, double th, double *phi) {
    phi[0] = (m.lam[i] - th) / m.scale;
    phi[1] = m.f1[i];
    phi[2] = m.f2[i];
    phi[3] = m.f3[i];
}

__device__ __forceinline__ double mlp(const double *P, const double *phi, double *z1, double *z2) {
#pragma unroll
    for (int a = 0; a < Hd; ++a) {
        double s = P[oB1 + a];
#pragma unroll
        for (int c = 0; c < F; ++c) s += P[oW1 + a * F + c] * phi[c];
        z1[a] = tanh(s);
    }
#pragma unroll
    for (int a = 0; a < Hd; ++a) {
        double s = P[oB2 + a];
#pragma unroll
        for (int b = 0; b < Hd; ++b) s += P[oW2 + a * Hd + b] * z1[b];
        z2[a] = tanh(s);
    }
    double f = P[oB3];
#pragma unroll
    for (int a = 0; a < Hd; ++a) f += P[oW3 + a] * z2[a];
    return f;
}

size_t chan_smem(int nmax, bool params) {
    return ((size_t)nmax * (nmax + 1) + 2 * (size_t)nmax * kCols + (params ? kLpParams : 0)) * sizeof(double);
}

__global__ void chan_apply_kernel(ChanPrec cp, const double *w, const double *R, long long ldr, const double *theta,
                                  int ncol, double *T, long long ldt, double *zraw) {
    extern __shared__ double sm[];
    const int c = blockIdx.x, n = cp.n[c], off = cp.off[c];
    const int j0 = blockIdx.y * kCols, nc = min(kCols, ncol - j0);
    // Q_c with an odd column stride sq (conflict-free reads down a column by consecutive modes)
    const int sq = n | 1;
    double *Q = sm, *Rc = Q + (size_t)cp.nmax * (cp.nmax + 1), *Z = Rc + (size_t)cp.nmax * kCols,
           *P = Z + (size_t)cp.nmax * kCols;
    const double *Qg = cp.Q + cp.qoff[c];
    const int *ix = cp.idx + off;
    for (int q = threadIdx.x; q < n * n; q += blockDim.x) Q[(q / n) * sq + q % n] = Qg[q];
    if (w)
        for (int q = threadIdx.x; q < kLpParams; q += blockDim.x) P[q] = w[q];
    for (int q = threadIdx.x; q < n * nc; q += blockDim.x) {
        const int p = q % n, jj = q / n;
        Rc[jj * n + p] = R[(size_t)(j0 + jj) * ldr + ix[p]];
    }
    __syncthreads();
    for (int q = threadIdx.x; q < n * nc; q += blockDim.x) {
        const int mq = q % n, jj = q / n;
        double s = 0.0;
        for (int p = 0; p < n; ++p) s += Q[mq * sq + p] * Rc[jj * n + p];
        const double th = theta[j0 + jj];
        const int mode = off + mq;
        const double zr = s / safe_den(cp.modes.lam[mode] - th);
        if (zraw) zraw[(size_t)(j0 + jj) * cp.modes.n + mode] = zr;
        double g = 1.0;
        if (w) {
            double phi[F], z1[Hd], z2[Hd];
            features(cp.modes, mode, th, phi);
            g += mlp(P, phi, z1, z2);
        }
        Z[jj * n + mq] = zr * g;
    }
    __syncthreads();
    for (int q = threadIdx.x; q < n * nc; q += blockDim.x) {
        const int p = q % n, jj = q / n;
        double s = 0.0;
        for (int mq = 0; mq < n; ++mq) s += Q[mq * sq + p] * Z[jj * n + mq];
        T[(size_t)(j0 + jj) * ldt + ix[p]] = s;
    }
}

__global__ void chan_back_kernel(ChanPrec cp, const double *G, long long ldg, const double *zraw, int ncol,
                                 double *delta) {
    extern __shared__ double sm[];
    const int c = blockIdx.x, n = cp.n[c], off = cp.off[c];
    const int j0 = blockIdx.y * kCols, nc = min(kCols, ncol - j0);
    const int sq = n | 1;
    double *Q = sm, *Gc = Q + (size_t)cp.nmax * (cp.nmax + 1);
    const double *Qg = cp.Q + cp.qoff[c];
    const int *ix = cp.idx + off;
    for (int q = threadIdx.x; q < n * n; q += blockDim.x) Q[(q / n) * sq + q % n] = Qg[q];
    for (int q = threadIdx.x; q < n * nc; q += blockDim.x) {
        const int p = q % n, jj = q / n;
        Gc[jj * n + p] = G[(size_t)(j0 + jj) * ldg + ix[p]];
    }
    __syncthreads();
    for (int q = threadIdx.x; q < n * nc; q += blockDim.x) {
        const int mq = q % n, jj = q / n;
        double s = 0.0;
        for (int p = 0; p < n; ++p) s += Q[mq * sq + p] * Gc[jj * n + p];
        const size_t o = (size_t)(j0 + jj) * cp.modes.n + off + mq;
        delta[o] = s * zraw[o];
    }
}

__global__ void lp_forward_kernel(LpModes m, const double *w, const double *theta, int ncol, double *gout) {
    __shared__ double P[kLpParams];
    for (int q = threadIdx.x; q < kLpParams; q += blockDim.x) P[q] = w[q];
    __syncthreads();
    const long long tot = (long long)m.n * ncol;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(t / m.n), i = (int)(t % m.n);
        double phi[F], z1[Hd], z2[Hd];
        features(m, i, theta[j], phi);
        gout[t] = 1.0 + mlp(P, phi, z1, z2);
    }
}

__global__ void __launch_bounds__(256) lp_grad_kernel(LpModes m, const double *w, const double *theta, int ncol,
                                                      const double *delta, double *gpart) {
    __shared__ double P[kLpParams];
    extern __shared__ double it[];  // [kChunk][kItem]
    for (int q = threadIdx.x; q < kLpParams; q += blockDim.x) P[q] = w[q];
    __syncthreads();
    const long long tot = (long long)m.n * ncol;
    const long long nchunk = (tot + kChunk - 1) / kChunk;
    const int p = threadIdx.x;
    double acc_a = 0.0, acc_b = 0.0;
    for (long long c = blockIdx.x; c < nchunk; c += gridDim.x) {
        if (p < kChunk) {
            double *q = it + (size_t)p * kItem;
            double *phi = q, *z1 = q + F, *z2 = z1 + Hd, *dl = z2 + Hd, *d2 = dl + 1, *d1 = d2 + Hd;
            const long long item = c * kChunk + p;
            if (item < tot) {
                const int j = (int)(item / m.n), i = (int)(item % m.n);
                features(m, i, theta[j], phi);
                mlp(P, phi, z1, z2);
                const double delta_f = delta[item];  // dL/df (g = 1 + f)
                dl[0] = delta_f;
#pragma unroll
                for (int a = 0; a < Hd; ++a) d2[a] = delta_f * P[oW3 + a] * (1.0 - z2[a] * z2[a]);
#pragma unroll
                for (int b = 0; b < Hd; ++b) {
                    double s = 0.0;
#pragma unroll
                    for (int a = 0; a < Hd; ++a) s += P[oW2 + a * Hd + b] * d2[a];
                    d1[b] = s * (1.0 - z1[b] * z1[b]);
                }
            } else {
                for (int u = 0; u < kItem; ++u) q[u] = 0.0;
            }
        }
        __syncthreads();
        {  // one thread per W2 entry
            const int a = p / Hd, b = p % Hd;
            for (int u = 0; u < kChunk; ++u) {
                const double *q = it + (size_t)u * kItem;
                acc_a += q[F + 2 * Hd + 1 + a] * q[F + b];  // d2[a] z1[b]
            }
        }
        if (p < Hd * F) {
            const int a = p / F, cc = p % F;
            for (int u = 0; u < kChunk; ++u) {
                const double *q = it + (size_t)u * kItem;
                acc_b += q[F + 3 * Hd + 1 + a] * q[cc];  // d1[a] phi[c]
            }
        } else if (p < Hd * F + Hd) {
            const int a = p - Hd * F;
            for (int u = 0; u < kChunk; ++u) acc_b += it[(size_t)u * kItem + F + 3 * Hd + 1 + a];  // d1[a]
        } else if (p < Hd * F + 2 * Hd) {
            const int a = p - Hd * F - Hd;
            for (int u = 0; u < kChunk; ++u) acc_b += it[(size_t)u * kItem + F + 2 * Hd + 1 + a];  // d2[a]
        } else if (p < Hd * F + 3 * Hd) {
            const int a = p - Hd * F - 2 * Hd;
            for (int u = 0; u < kChunk; ++u) {
                const double *q = it + (size_t)u * kItem;
                acc_b += q[F + 2 * Hd] * q[F + Hd + a];  // delta z2[a]
            }
        } else if (p == Hd * F + 3 * Hd) {
            for (int u = 0; u < kChunk; ++u) acc_b += it[(size_t)u * kItem + F + 2 * Hd];  // delta
        }
        __syncthreads();
    }
    double *g = gpart + (size_t)blockIdx.x * kLpParams;
    g[oW2 + p] = acc_a;  // 256 threads <-> W2
    if (p < Hd * F) g[oW1 + p] = acc_b;
    else if (p < Hd * F + Hd) g[oB1 + p - Hd * F] = acc_b;
    else if (p < Hd * F + 2 * Hd) g[oB2 + p - Hd * F - Hd] = acc_b;
    else if (p < Hd * F + 3 * Hd) g[oW3 + p - Hd * F - 2 * Hd] = acc_b;
    else if (p == Hd * F + 3 * Hd) g[oB3] = acc_b;
}

__global__ void lp_grad_reduce_kernel(const double *gpart, int nb, double *grad) {
    for (int p = threadIdx.x; p < kLpParams; p += blockDim.x) {
        double s = 0.0;
        for (int b = 0; b < nb; ++b) s += gpart[(size_t)b * kLpParams + p];
        grad[p] = s;
    }
}

__global__ void lp_adam_kernel(double *w, const double *grad, double *m, double *v, int step, double lr) {
    const double b1 = 0.9, b2 = 0.999, eps = 1.0e-8;
    const double c1 = 1.0 - pow(b1, (double)step), c2 = 1.0 - pow(b2, (double)step);
    for (int p = threadIdx.x; p < kLpParams; p += blockDim.x) {
        const double g = grad[p];
        const double mm = b1 * m[p] + (1.0 - b1) * g, vv = b2 * v[p] + (1.0 - b2) * g * g;
        m[p] = mm;
        v[p] = vv;
        w[p] -= lr * (mm / c1) / (sqrt(vv / c2) + eps);
    }
}

__global__ void lp_pair_sums_kernel(const double *T, const double *PT, const double *E, long long ld, int n,
                                    double *sums) {
    const int j = blockIdx.x;
    const double *t = T + (size_t)j * ld, *pt = PT + (size_t)j * ld, *e = E + (size_t)j * ld;
    double te = 0.0, pp = 0.0, ee = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        te += t[i] * e[i];
        pp += pt[i] * pt[i];
        ee += e[i] * e[i];
    }
    __shared__ double red[32];
    te = block_sum(te, red);
    pp = block_sum(pp, red);
    ee = block_sum(ee, red);
    if (threadIdx.x == 0) {
        sums[3 * j] = te;
        sums[3 * j + 1] = pp;
        sums[3 * j + 2] = ee;
    }
}

__global__ void lp_coef_kernel(const double *sums, int npair, double *coef, double *loss) {
    __shared__ double red[32];
    double lsum = 0.0, nv = 0.0;
    for (int j = threadIdx.x; j < npair; j += blockDim.x) {
        const double te = sums[3 * j], pp = sums[3 * j + 1], ee = sums[3 * j + 2];
        const bool ok = (pp > 0.0 && ee > 0.0 && isfinite(te) && isfinite(pp));
        if (ok) {
            lsum += 1.0 - te * te / (pp * ee);
            nv += 1.0;
        }
    }
    lsum = block_sum(lsum, red);
    nv = block_sum(nv, red);
    const double inv = nv > 0.0 ? 1.0 / nv : 0.0;
    for (int j = threadIdx.x; j < npair; j += blockDim.x) {
        const double te = sums[3 * j], pp = sums[3 * j + 1], ee = sums[3 * j + 2];
        const bool ok = (pp > 0.0 && ee > 0.0 && isfinite(te) && isfinite(pp));
        coef[2 * j] = ok ? -2.0 * te / (pp * ee) * inv : 0.0;
        coef[2 * j + 1] = ok ? 2.0 * te * te / (pp * pp * ee) * inv : 0.0;
    }
    if (threadIdx.x == 0) loss[0] = lsum * inv;
}

__global__ void lp_dldt_kernel(const double *E, const double *PT, long long ld, int n, int npair, const double *coef,
                               double *G) {
    const long long tot = (long long)ld * npair;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(t / ld), i = (int)(t % ld);
        G[t] = (i < n) ? coef[2 * j] * E[t] + coef[2 * j + 1] * PT[t] : 0.0;
    }
}

cudaError_t set_smem(const void *fn, size_t bytes) {
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

}  // namespace

cudaError_t launch_chan_apply(const ChanPrec &cp, const double *w, const double *R, long long ldr,
                              const double *theta, int ncol, double *T, long long ldt, double *zraw,
                              cudaStream_t st) {
    if (cp.nch <= 0 || ncol <= 0) return cudaSuccess;
    const size_t smem = chan_smem(cp.nmax, true);
    if (smem > 220 * 1024) return cudaErrorInvalidValue;
    cudaError_t e = set_smem((const void *)chan_apply_kernel, smem);
    if (e != cudaSuccess) return e;
    DVR3D_COUNT_LAUNCH(1);
    chan_apply_kernel<<<dim3(cp.nch, (ncol + kCols - 1) / kCols), 128, smem, st>>>(cp, w, R, ldr, theta, ncol, T, ldt,
                                                                                 zraw);
    return cudaGetLastError();
}

cudaError_t launch_chan_back(const ChanPrec &cp, const double *G, long long ldg, const double *zraw, int ncol,
                             double *delta, cudaStream_t st) {
    if (cp.nch <= 0 || ncol <= 0) return cudaSuccess;
    const size_t smem = chan_smem(cp.nmax, false);
    if (smem > 220 * 1024) return cudaErrorInvalidValue;
    cudaError_t e = set_smem((const void *)chan_back_kernel, smem);
    if (e != cudaSuccess) return e;
    DVR3D_COUNT_LAUNCH(1);
    chan_back_kernel<<<dim3(cp.nch, (ncol + kCols - 1) / kCols), 128, smem, st>>>(cp, G, ldg, zraw, ncol, delta);
    return cudaGetLastError();
}

cudaError_t launch_lp_forward(const LpModes &m, const double *w, const double *theta, int ncol, double *gout,
                              cudaStream_t st) {
    if (m.n <= 0 || ncol <= 0) return cudaSuccess;
    const long long tot = (long long)m.n * ncol;
    DVR3D_COUNT_LAUNCH(1);
    lp_forward_kernel<<<(unsigned)std::min<long long>((tot + 255) / 256, 1184), 256, 0, st>>>(m, w, theta, ncol, gout);
    return cudaGetLastError();
}

size_t lp_grad_work_doubles() { return (size_t)kGradGrid * kLpParams; }

cudaError_t lp_mlp_grad(const LpModes &m, const double *w, const double *theta, int ncol, const double *delta,
                        double *grad, double *work, cudaStream_t st) {
    const size_t smem = (size_t)kChunk * kItem * sizeof(double);
    cudaError_t e = set_smem((const void *)lp_grad_kernel, smem);
    if (e != cudaSuccess) return e;
    DVR3D_COUNT_LAUNCH(2);
    lp_grad_kernel<<<kGradGrid, 256, smem, st>>>(m, w, theta, ncol, delta, work);
    lp_grad_reduce_kernel<<<1, 384, 0, st>>>(work, kGradGrid, grad);
    return cudaGetLastError();
}

cudaError_t lp_adam_step(double *w, const double *grad, double *mom, double *vel, int step, double lr,
                         cudaStream_t st) {
    DVR3D_COUNT_LAUNCH(1);
    lp_adam_kernel<<<1, 384, 0, st>>>(w, grad, mom, vel, step, lr);
    return cudaGetLastError();
}

cudaError_t launch_lp_pair_terms(const double *T, const double *PT, const double *E, long long ld, int n,
                                 int npair, double *sums, double *coef, double *loss, cudaStream_t st) {
    DVR3D_COUNT_LAUNCH(2);
    lp_pair_sums_kernel<<<npair, 256, 0, st>>>(T, PT, E, ld, n, sums);
    lp_coef_kernel<<<1, 256, 0, st>>>(sums, npair, coef, loss);
    return cudaGetLastError();
}

cudaError_t launch_lp_dldt(const double *E, const double *PT, long long ld, int n, int npair, const double *coef,
                           double *G, cudaStream_t st) {
    const long long tot = ld * npair;
    DVR3D_COUNT_LAUNCH(1);
    lp_dldt_kernel<<<(unsigned)std::min<long long>((tot + 255) / 256, 1184), 256, 0, st>>>(E, PT, ld, n, npair, coef, G);
    return cudaGetLastError();
}

}  // namespace dvr3d
