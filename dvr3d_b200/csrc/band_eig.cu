// band_eig.cu -- symmetric band matrix -> tridiagonal by bulge chasing, and the
// back-transformation of eigenvectors, for the projected matrix of the block Krylov solve.
//
// The block Lanczos recurrence makes T = Q^T M Q block tridiagonal: with full
// reorthogonalisation the entries more than one block (b) away from the diagonal are
// rounding-level reorthogonalisation coefficients, so T is a band matrix of half-bandwidth
// b. Instead of the dense one-stage reduction (O(m^2) grid-synchronised column steps) the
// band is chased to tridiagonal form (Schwarz / Lang successive bulge chasing, the
// "band to tridiagonal" stage of two-stage reductions):
//   sweep j, task 0: reflector H_0 annihilating A[j+2 : j+b+1, j]; H_0 applied from both
//                    sides to the diagonal block D_0 (rows/cols R_0 = [j+1, j+b]) and from
//                    the right to the block below it, O_1 = A[R_1, R_0] (which fills: the
//                    bulge);
//   task s >= 1:     H_s annihilates the first column of the bulge O_s below its first
//                    entry, is applied from the left to the rest of O_s, from both sides to
//                    D_s and from the right to O_{s+1}; the remainder of the bulge is
//                    eliminated by later sweeps.
// One CTA owns a whole sweep (five warps with fixed roles, 32 x 32 blocks in shared memory,
// lane = row), keeping O_{s+1} between its tasks. Sweep j+1 may start task s once sweep j has
// written the beta of its task s + 2 (the only entry the two share), published through
// per-sweep progress counters with release / acquire ordering and bounded waits.
// Back-transformation: Q = prod over sweeps (in order) of prod over tasks of H; the
// reflectors of one sweep act on disjoint rows, so a CTA holding a slab of eigenvector
// columns in shared memory applies sweep after sweep (last first), its warps taking the
// tasks of a sweep in parallel.
#include <algorithm>

#include "band_eig.cuh"
#include "common.cuh"

namespace dvr3d {

namespace {

constexpr int kBW = kBandMaxBw;
constexpr int kTS = kBW + 1;            // shared-memory row stride of a block
constexpr int kChaseThreads = 160;      // five warps per sweep in flight
constexpr int kBlk = kBW * kTS;         // doubles of one 32 x 32 block in shared memory
constexpr size_t kChaseSmem = ((size_t)6 * kBlk + 3 * kBW) * sizeof(double);
constexpr unsigned long long kSpinLimit = 1ull << 24;
constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_u32(unsigned *p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__host__ __device__ __forceinline__ int band_ntask(int n, int b, int j) { return (n - 2 - j) / b + 1; }

__global__ void band_prepare_kernel(double *A, long long lda, int n, int b, unsigned long long *maxbits2) {
    // column j per block-row of threads; rows i > j
    double dropped = 0.0, inside = 0.0;
    const long long tot = (long long)n * n;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(t / n), i = (int)(t % n);
        if (i < j) continue;
        double *p = A + (size_t)j * lda + i;
        const double a = fabs(*p);
        if (i - j <= b) inside = fmax(inside, a);
        else {
            dropped = fmax(dropped, a);
            if (i - j <= 2 * b) *p = 0.0;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        dropped = fmax(dropped, __shfl_xor_sync(kFull, dropped, o));
        inside = fmax(inside, __shfl_xor_sync(kFull, inside, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(maxbits2, (unsigned long long)__double_as_longlong(dropped));
        atomicMax(maxbits2 + 1, (unsigned long long)__double_as_longlong(inside));
    }
}

// Householder reflector of x (lanes 0..L-1): H x = beta e_0, v[0] = 1.
__device__ __forceinline__ void warp_house(double x, int lane, int L, double &v, double &tau, double &beta) {
    const double alpha = __shfl_sync(kFull, x, 0);
    const double sig = warp_sum((lane >= 1 && lane < L) ? x * x : 0.0);
    tau = 0.0;
    beta = alpha;
    v = (lane == 0) ? 1.0 : 0.0;
    if (sig != 0.0) {
        beta = -copysign(sqrt(alpha * alpha + sig), alpha);
        tau = (beta - alpha) / beta;
        const double sc = 1.0 / (alpha - beta);
        v = (lane == 0) ? 1.0 : ((lane < L) ? x * sc : 0.0);
    }
}

// One CTA per sweep in flight, five warps with fixed roles per task s:
//   warp 0: the reflector (from column j or the bulge's first column); its beta is written
//           and the task published to the next sweep at once (the next sweep's task s-2,
//           which this publication releases, shares only that entry with task s); then
//           O_s <- H O_s, written back;
//   warp 1: D_s <- H D_s H, written back (lower triangle);
//   warp 2: O_{s+1} <- O_{s+1} H, kept in shared memory for task s+1;
//   warps 3, 4: wait for the previous sweep and load task s+1's O_{s+2} and D_{s+1}.
// Warps 0-2 start after the reflector is in shared memory; all five meet at the end of the
// task, so a publication also covers everything of the earlier tasks. The last task of a
// sweep is published only when all its parts are written.
__global__ void __launch_bounds__(kChaseThreads) band_chase_kernel(BandTri t) {
    extern __shared__ double sm[];
    double *Ob = sm;                   // [2] O_s (held from the previous task) / O_{s+1}
    double *Dr = sm + 2 * kBlk;        // [2] D_s as loaded (lower triangle, zeros elsewhere)
    double *Orw = sm + 4 * kBlk;       // [2] O_{s+1} as loaded
    double *Xr = sm + 6 * kBlk;        // column j below the diagonal (task 0)
    double *vsm = Xr + kBW;            // reflector
    double *wsm = vsm + kBW;           // w of the diagonal-block update
    __shared__ double s_tau, s_beta;
    __shared__ int s_abort;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int n = t.n, b = t.b;
    const long long ld = t.lda;
    const unsigned long long spin_limit = t.wait_limit ? t.wait_limit : kSpinLimit;
    double *A = t.A;
    for (int q = tid; q < 6 * kBlk + 3 * kBW; q += kChaseThreads) sm[q] = 0.0;
    if (tid == 0) s_abort = 0;
    __syncthreads();
    long long pc[5] = {0, 0, 0, 0, 0};
    long long tlast = clock64();
    auto mark = [&](int ph) {
        if (t.prof) {
            const long long now = clock64();
            pc[ph] += now - tlast;
            tlast = now;
        }
    };
    // warps 3 (which = 0: O_{s+1}, and column j for task 0) and 4 (which = 1: D_s): wait
    // until sweep j-1 has published `need` tasks, then load task s's block
    auto load_task = [&](int j, int s, int buf, int need, int which) {
        if (j > 0) {
            int ok = 1;
            if (lane == 0) {
                unsigned long long spins = 0;
                while (ld_acquire_u32(t.progress + j - 1) < (unsigned)need) {
                    if (++spins > spin_limit) {
                        atomicExch(t.err, (int)kDevBarrierTimeout);
                        ok = 0;
                        break;
                    }
                    if ((spins & 255ull) == 0 && *(volatile int *)t.err != 0) {
                        ok = 0;
                        break;
                    }
                    if (spins > 32) __nanosleep(32);
                }
            }
            ok = __shfl_sync(kFull, ok, 0);
            if (!ok) {
                if (lane == 0) s_abort = 1;
                return;
            }
        }
        __syncwarp();
        const int r0 = j + 1 + s * b, L = min(b, n - r0);
        const int r1 = r0 + b, L1 = (r1 < n) ? min(b, n - r1) : 0;
        const int rl = min(r0 + lane, n - 1), rl1 = min(r1 + lane, n - 1);
        double val[kBW];
        if (which == 1) {
#pragma unroll
            for (int c = 0; c < kBW; ++c) {
                const double a0 = __ldcg(A + (size_t)min(r0 + c, n - 1) * ld + rl);
                val[c] = (c < L && lane >= c && lane < L) ? a0 : 0.0;
            }
            double *D = Dr + buf * kBlk;
#pragma unroll
            for (int c = 0; c < kBW; ++c) D[lane * kTS + c] = val[c];
        } else {
#pragma unroll
            for (int c = 0; c < kBW; ++c) {
                const double a1 = __ldcg(A + (size_t)min(r0 + c, n - 1) * ld + rl1);
                val[c] = (c < b && lane < L1) ? a1 : 0.0;
            }
            if (s == 0) {
                const double xv = __ldcg(A + (size_t)j * ld + rl);
                Xr[lane] = (lane < L) ? xv : 0.0;
            }
            double *O = Orw + buf * kBlk;
#pragma unroll
            for (int c = 0; c < kBW; ++c) O[lane * kTS + c] = val[c];
        }
    };
    for (int j = blockIdx.x; j <= n - 3; j += gridDim.x) {
        const int nt = band_ntask(n, b, j);
        const int ntp = (j > 0) ? band_ntask(n, b, j - 1) : 0;
        if (warp >= 3) load_task(j, 0, 0, min(3, ntp), warp - 3);
        __syncthreads();
        if (s_abort) return;
        mark(0);
        for (int s = 0; s < nt; ++s) {
            const int cur = s & 1;
            const int r0 = j + 1 + s * b, L = min(b, n - r0);
            const int r1 = r0 + b, L1 = (r1 < n) ? min(b, n - r1) : 0;
            double *Oc = Ob + cur * kBlk, *On = Ob + (cur ^ 1) * kBlk;
            const double *Dc = Dr + cur * kBlk, *Oraw = Orw + cur * kBlk;
            if (warp == 0) {
                const double x = (s == 0) ? Xr[lane] : ((lane < L) ? Oc[lane * kTS] : 0.0);
                double v, tau, beta;
                warp_house(x, lane, L, v, tau, beta);
                vsm[lane] = v;
                // beta at once, then the publication (the rest of O_s follows below). The
                // release store is cumulative over the earlier tasks' writes of every warp,
                // which the end-of-task barrier ordered before it.
                if (lane == 0) {
                    s_tau = tau;
                    s_beta = beta;
                    if (s == 0) A[(size_t)j * ld + r0] = beta;
                    else A[(size_t)(r0 - b) * ld + r0] = beta;
                    if (s + 1 < nt) st_release_u32(t.progress + j, (unsigned)(s + 1));
                    t.taus[(size_t)j * t.ntmax + s] = tau;
                }
                t.vs[((size_t)j * t.ntmax + s) * kBW + lane] = v;
            }
            __syncthreads();
            mark(1);
            const double tau = s_tau;
            const double vme = vsm[lane];
            if (warp == 0) {
                if (s == 0) {
                    if (lane < L) A[(size_t)j * ld + r0 + lane] = (lane == 0) ? s_beta : 0.0;
                } else {
                    // O_s <- H O_s (lane = column; v is zero past row L)
                    double z0 = 0.0, z1 = 0.0, z2 = 0.0, z3 = 0.0;
#pragma unroll
                    for (int l = 0; l < kBW; l += 4) {
                        z0 += vsm[l] * Oc[l * kTS + lane];
                        z1 += vsm[l + 1] * Oc[(l + 1) * kTS + lane];
                        z2 += vsm[l + 2] * Oc[(l + 2) * kTS + lane];
                        z3 += vsm[l + 3] * Oc[(l + 3) * kTS + lane];
                    }
                    const double z = (lane >= 1 && lane < b) ? tau * ((z0 + z1) + (z2 + z3)) : 0.0;
#pragma unroll
                    for (int l = 0; l < kBW; ++l) Oc[l * kTS + lane] -= vsm[l] * z;
                    __syncwarp();
                    if (lane < L) Oc[lane * kTS] = (lane == 0) ? s_beta : 0.0;
                    __syncwarp();
                    if (lane < L) {
                        double *dst = A + (size_t)(r0 - b) * ld + r0 + lane;
                        for (int c = 0; c < b; ++c) dst[(size_t)c * ld] = Oc[lane * kTS + c];
                    }
                }
            } else if (warp == 1) {
                if (tau != 0.0) {
                    // y_l = sum_c (D[l][c] + D[c][l]) v_c - D[l][l] v_l
                    double y0 = 0.0, y1 = 0.0, y2 = 0.0, y3 = 0.0;
#pragma unroll
                    for (int c = 0; c < kBW; c += 4) {
                        y0 += (Dc[lane * kTS + c] + Dc[c * kTS + lane]) * vsm[c];
                        y1 += (Dc[lane * kTS + c + 1] + Dc[(c + 1) * kTS + lane]) * vsm[c + 1];
                        y2 += (Dc[lane * kTS + c + 2] + Dc[(c + 2) * kTS + lane]) * vsm[c + 2];
                        y3 += (Dc[lane * kTS + c + 3] + Dc[(c + 3) * kTS + lane]) * vsm[c + 3];
                    }
                    const double y = ((y0 + y1) + (y2 + y3)) - Dc[lane * kTS + lane] * vme;
                    const double K = warp_sum(vme * y);
                    const double w = tau * y - 0.5 * tau * tau * K * vme;
                    wsm[lane] = w;
                    __syncwarp();
                    if (lane < L) {
                        double *dst = A + (size_t)r0 * ld + r0 + lane;
#pragma unroll
                        for (int c = 0; c < kBW; ++c)
                            if (c <= lane) dst[(size_t)c * ld] = Dc[lane * kTS + c] - (vme * wsm[c] + w * vsm[c]);
                    }
                }
            } else if (warp == 2) {
                if (L1 > 0) {
                    double u0 = 0.0, u1 = 0.0, u2 = 0.0, u3 = 0.0;
#pragma unroll
                    for (int c = 0; c < kBW; c += 4) {
                        u0 += Oraw[lane * kTS + c] * vsm[c];
                        u1 += Oraw[lane * kTS + c + 1] * vsm[c + 1];
                        u2 += Oraw[lane * kTS + c + 2] * vsm[c + 2];
                        u3 += Oraw[lane * kTS + c + 3] * vsm[c + 3];
                    }
                    const double u = tau * ((u0 + u1) + (u2 + u3));
#pragma unroll
                    for (int c = 0; c < kBW; ++c) On[lane * kTS + c] = Oraw[lane * kTS + c] - u * vsm[c];
                }
            } else {
                if (s + 1 < nt) load_task(j, s + 1, cur ^ 1, min(s + 4, ntp), warp - 3);
            }
            mark(2);
            __syncthreads();
            if (s_abort) return;
            mark(3);
            if (s + 1 == nt && tid == 0) {
                __threadfence();
                st_release_u32(t.progress + j, (unsigned)nt);
            }
        }
    }
    if (t.prof && tid == 0) {
#pragma unroll
        for (int q = 0; q < 5; ++q) atomicAdd(reinterpret_cast<unsigned long long *>(t.prof + q), (unsigned long long)pc[q]);
    }
}

__global__ void band_diag_kernel(const double *A, long long lda, int n, double *d, double *e) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    d[i] = A[(size_t)i * lda + i];
    e[i] = (i + 1 < n) ? A[(size_t)i * lda + i + 1] : 0.0;
}

// Back-transformation, COLS eigenvector columns per CTA held in shared memory (column c at
// zs + c ldzs, ldzs = 1 mod 16 so the lanes' rows and columns spread over the banks).
// Sweeps are applied last first; the tasks of one sweep act on disjoint rows and are split
// over the 8 warps (task w + 8 k of a chunk of kChunkTasks). In a warp, lane (rg, c) takes
// column c and rows COLS rg .. COLS rg + COLS - 1 of the reflector's window: COLS products,
// a shuffle sum over the 32 / COLS row groups, COLS updates. The reflectors of the next
// chunk are copied into shared memory (cp.async) while the current chunk is applied.
constexpr int kChunkTasks = 96;

__device__ __forceinline__ void cp_async8(double *dst, const double *src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}

template <int COLS>
__global__ void __launch_bounds__(256) band_bt_kernel(BandTri t, double *Z, long long ldz, int nev, int ldzs) {
    extern __shared__ double sm[];
    double *zs = sm;
    double *vb = sm + (size_t)COLS * ldzs;       // [2][kChunkTasks][kBW]
    double *tb = vb + 2 * kChunkTasks * kBW;     // [2][kChunkTasks]
    const int n = t.n, b = t.b;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int cc = lane % COLS, rg = lane / COLS;
    const int c0 = blockIdx.x * COLS;
    const int ncol = min(COLS, nev - c0);
    for (int q = tid; q < COLS * n; q += blockDim.x) {
        const int c = q / n, r = q - c * n;
        zs[(size_t)c * ldzs + r] = (c < ncol) ? Z[(size_t)(c0 + c) * ldz + r] : 0.0;
    }
    auto stage = [&](int j, int base, int buf) {
        const int cnt = min(kChunkTasks, band_ntask(n, b, j) - base);
        const double *vsrc = t.vs + ((size_t)j * t.ntmax + base) * kBW;
        double *vd = vb + (size_t)buf * kChunkTasks * kBW;
        for (int q = tid; q < cnt * kBW; q += blockDim.x) cp_async8(vd + q, vsrc + q);
        const double *tsrc = t.taus + (size_t)j * t.ntmax + base;
        double *td = tb + buf * kChunkTasks;
        for (int q = tid; q < cnt; q += blockDim.x) cp_async8(td + q, tsrc + q);
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    int j = n - 3, base = 0, buf = 0;
    if (j >= 0) stage(j, base, buf);
    while (j >= 0) {
        asm volatile("cp.async.wait_group 0;" ::: "memory");
        __syncthreads();  // chunk (j, base) staged; the previous chunk's updates are done
        const int cj = j, cbase = base, cbuf = buf;
        base += kChunkTasks;
        if (base >= band_ntask(n, b, j)) {
            --j;
            base = 0;
        }
        buf ^= 1;
        if (j >= 0) stage(j, base, buf);
        const double *vd = vb + (size_t)cbuf * kChunkTasks * kBW;
        const double *td = tb + cbuf * kChunkTasks;
        const int nt = band_ntask(n, b, cj);
        for (int s = cbase + warp; s < nt && s < cbase + kChunkTasks; s += 8) {
            const double tau = td[s - cbase];
            if (tau == 0.0) continue;
            const int r0 = cj + 1 + s * b;
            const double *v = vd + (size_t)(s - cbase) * kBW + rg * COLS;
            double vv[COLS], zz[COLS];
            double part = 0.0;
#pragma unroll
            for (int i = 0; i < COLS; ++i) {
                const int r = min(r0 + rg * COLS + i, n - 1);
                vv[i] = v[i];
                zz[i] = zs[(size_t)cc * ldzs + r];
                part += vv[i] * zz[i];
            }
#pragma unroll
            for (int o = COLS; o < 32; o <<= 1) part += __shfl_xor_sync(kFull, part, o);
            const double f = tau * part;
#pragma unroll
            for (int i = 0; i < COLS; ++i) {
                const int r = r0 + rg * COLS + i;
                if (vv[i] != 0.0 && r < n) zs[(size_t)cc * ldzs + r] = zz[i] - f * vv[i];
            }
        }
    }
    __syncthreads();
    for (int q = tid; q < COLS * n; q += blockDim.x) {
        const int c = q / n, r = q - c * n;
        if (c < ncol) Z[(size_t)(c0 + c) * ldz + r] = zs[(size_t)c * ldzs + r];
    }
}

template <int COLS>
cudaError_t launch_bt(const BandTri &t, double *Z, long long ldz, int nev, int ldzs, size_t smem, cudaStream_t st) {
    cudaError_t e = cudaFuncSetAttribute(band_bt_kernel<COLS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    DVR3D_COUNT_LAUNCH(1);
    band_bt_kernel<COLS><<<(unsigned)((nev + COLS - 1) / COLS), 256, smem, st>>>(t, Z, ldz, nev, ldzs);
    return cudaGetLastError();
}

}  // namespace

size_t band_reflector_doubles(int n, int b) {
    const size_t nt = (size_t)((n - 2) / std::max(b, 1) + 1);
    return (size_t)std::max(n - 2, 1) * nt * kBW;
}

size_t band_tau_doubles(int n, int b) {
    const size_t nt = (size_t)((n - 2) / std::max(b, 1) + 1);
    return (size_t)std::max(n - 2, 1) * nt;
}

cudaError_t launch_band_prepare(double *A, long long lda, int n, int b, unsigned long long *maxbits2,
                                cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(maxbits2, 0, 2 * sizeof(unsigned long long), st);
    if (e != cudaSuccess) return e;
    DVR3D_COUNT_LAUNCH(1);
    band_prepare_kernel<<<592, 256, 0, st>>>(A, lda, n, b, maxbits2);
    return cudaGetLastError();
}

cudaError_t launch_band_chase(BandTri &t, cudaStream_t st) {
    if (t.b < 1 || t.b > kBW || t.n < 3) return cudaErrorInvalidValue;
    t.ntmax = band_ntask(t.n, t.b, 0);
    cudaError_t e = cudaMemsetAsync(t.progress, 0, sizeof(unsigned) * t.n, st);
    if (e != cudaSuccess) return e;
    const size_t smem = kChaseSmem;
    e = cudaFuncSetAttribute(band_chase_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    // one CTA per sweep in flight: sweeps start about three tasks apart and a CTA is busy
    // for ntask tasks, so ntask / 3 plus slack keeps every sweep's successor supplied
    int grid = std::min(t.n - 2, std::max(8, t.ntmax / 2 + 8));
    int dev = 0, nsm = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, band_chase_kernel, kChaseThreads, smem);
    grid = std::max(1, std::min(grid, nsm * std::max(per, 1)));
    void *args[] = {&t};
    DVR3D_COUNT_LAUNCH(1);
    e = cudaLaunchCooperativeKernel((void *)band_chase_kernel, dim3(grid), dim3(kChaseThreads), args, smem, st);
    if (e != cudaSuccess) return e;
    DVR3D_COUNT_LAUNCH(1);
    band_diag_kernel<<<(t.n + 255) / 256, 256, 0, st>>>(t.A, t.lda, t.n, t.d, t.e);
    return cudaGetLastError();
}

cudaError_t launch_band_backtransform(const BandTri &t, double *Z, long long ldz, int nev, cudaStream_t st) {
    if (nev <= 0 || t.n < 3) return cudaSuccess;
    int optin = 0, dev = 0, nsm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const int ldzs = (t.n + 15) / 16 * 16 + 1;
    const size_t fixed = (size_t)2 * kChunkTasks * (kBW + 1) * sizeof(double);
    auto need = [&](int cols) { return fixed + (size_t)cols * ldzs * sizeof(double); };
    // widest slab that fits, but no wider than keeps every SM busy
    int cols = 8;
    while (cols > 1 && (need(cols) > (size_t)optin || (nev + cols - 1) / cols < nsm)) cols /= 2;
    if (need(cols) > (size_t)optin) return cudaErrorInvalidValue;
    switch (cols) {
        case 8: return launch_bt<8>(t, Z, ldz, nev, ldzs, need(8), st);
        case 4: return launch_bt<4>(t, Z, ldz, nev, ldzs, need(4), st);
        case 2: return launch_bt<2>(t, Z, ldz, nev, ldzs, need(2), st);
        default: return launch_bt<1>(t, Z, ldz, nev, ldzs, need(1), st);
    }
}

}  // namespace dvr3d
