// eig_dense.cu -- FP64 eigensolver for the final N x N Hamiltonian (lowest K levels).
//
// Replaces diag3d -> diag -> dsyev('V','L') of the reference (:2661-2764, :2638-2659) for
// the plain FP64 path. Same structure as the batched solver (Householder reduction,
// bisection, inverse iteration, back-transformation) but spread over the whole GPU:
//   - the reduction is blocked like LAPACK's dsytrd/dlatrd: a cooperative kernel forms
//     the 32 reflectors of a panel (one symmetric product over the lower triangle of the
//     trailing matrix per column, in 64x64 tiles with deterministic partial sums and four
//     bounded grid barriers per column), then a DMMA SYR2K updates the trailing matrix;
//   - eigenvalues by multisection: one warp per wanted eigenvalue, 32 Sturm counts per
//     pass, the interval shrinks 33x per pass;
//   - inverse iteration one thread per cluster of close eigenvalues;
//   - back-transformation by the stored reflectors, one warp per 4 eigenvectors.
#include <algorithm>
#include <cfloat>
#include <cmath>

#include "common.cuh"
#include "eig_dense.cuh"
#include "gemm64.cuh"
#include "tridiag_dev.cuh"

namespace dvr3d {

namespace {

constexpr int TB = 64;          // symmetric tile edge
constexpr int TS = TB + 1;      // shared-memory column stride (conflict-free transposed reads)
constexpr int kPnThreads = 256;
constexpr int kMaxNb = 64;
constexpr int kPw = 32;         // panel width of the reduction (columns per panel)

constexpr int kChunk = 256;     // rows owned by one owner CTA (one row per thread)

// Optional phase timers: CTA 0 accumulates SM clock cycles spent in each phase
// (prof[0..5]: column update, reflector, symmetric product, reduction, w, exit).
#define PROF_MARK(ph)                                                   \
    do {                                                                \
        if (t.prof && cta == 0 && tid == 0) {                          \
            const long long now_ = clock64();                           \
            if (prof_last_ >= 0) t.prof[prof_ph_] += now_ - prof_last_; \
            prof_last_ = now_;                                          \
            prof_ph_ = (ph);                                            \
        }                                                               \
    } while (0)

// One panel of the blocked Householder reduction (the dlatrd scheme: columns are formed
// from the panel-start matrix plus the rank-2 corrections V W^T + W V^T of the panel's
// earlier columns; the trailing matrix itself is updated once per panel by syr2k).
// Work split: every CTA takes 64x64 lower tiles of the symmetric product, the V/W dot
// products and rows of the reduction; the first NO = ceil(n/256) CTAs also own 256 rows
// each for the column update, so the norm is a sum over NO partials only.
// Per column three bounded grid barriers separate: column update (with the previous
// column's w) + norm | reflector, symmetric product (deterministic per-tile partial sums),
// V^T v and W^T v | reduction of the partials into p = tau y and p.v.
__global__ void __launch_bounds__(kPnThreads, 3) dense_panel_kernel(DenseTri t) {
    const int n = t.n, NT = t.NT;
    const long long ld = t.lda;
    double *A = t.A;
    const int G = gridDim.x, cta = blockIdx.x, tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int NO = (n + kChunk - 1) / kChunk;
    const bool owner = cta < NO;
    const int r_own = cta * kChunk + tid;  // the row this thread owns (if owner)
    extern __shared__ double dsm[];
    double *cache = dsm;                              // t.cache_tiles resident tiles (panel-start values)
    double *S = dsm + (size_t)t.cache_tiles * TB * TS;  // scratch tile for the streamed path
    __shared__ double vI[TB], vJ[TB];
    __shared__ double red[32];
    __shared__ double rsum[4][TB];
    __shared__ double rsJ[4][TB];
    __shared__ double s_corr[2 * kMaxNb];
    __shared__ double s_red4[4][2 * kPw];
    __shared__ double s_tau, s_scal, s_a2;
    const int nbmax = t.nbmax;
    double *part_n = t.part;                  // [NO] partial norms of the column
    double *part_d = t.part + G;              // [G] partial p.v
    double *part_q = t.part + 2 * G;          // [NO][2 nbmax] V^T v, W^T v
    long long prof_last_ = -1;
    int prof_ph_ = 0;
    // resident mode: this CTA's lower tiles of the trailing matrix (fixed for the panel: the
    // reduction forms columns from the panel-start matrix) are read once into shared memory;
    // tiles beyond the cache are streamed from global memory per column as below
    const int t0s = (t.j0 + 1) / TB;
    const long long ntiles_s = (long long)(NT - t0s) * (NT - t0s + 1) / 2;
    auto decode_rel = [&](long long tt, int base, int &Io, int &Jo) {
        int li = (int)((sqrt(8.0 * (double)tt + 1.0) - 1.0) * 0.5);
        while ((long long)li * (li + 1) / 2 > tt) --li;
        while ((long long)(li + 1) * (li + 2) / 2 <= tt) ++li;
        Io = base + li;
        Jo = base + (int)(tt - (long long)li * (li + 1) / 2);
    };
    if (t.cache_tiles > 0) {
        int slot = 0;
        for (long long tt = cta; tt < ntiles_s && slot < t.cache_tiles; tt += G, ++slot) {
            int I, J;
            decode_rel(tt, t0s, I, J);
            double *Sc = cache + (size_t)slot * TB * TS;
            const int r0 = I * TB, c0 = J * TB;
            for (int q = tid; q < TB * TB; q += kPnThreads) {
                const int c = q / TB, r = q % TB;
                const int gr = r0 + r, gc = c0 + c;
                Sc[c * TS + r] = (gr < n && gc < n) ? __ldcg(A + (size_t)gc * ld + gr) : 0.0;
            }
            if (I == J) {
                __syncthreads();
                for (int q = tid; q < TB * TB; q += kPnThreads) {
                    const int c = q / TB, r = q % TB;
                    if (r < c) Sc[c * TS + r] = Sc[r * TS + c];
                }
            }
        }
        __syncthreads();
    }
    // w of the previous column: w = p - (tau/2)(p.v) v, with p (ybuf) and the partial p.v of
    // every CTA (part_d) from its reduction phase
    auto prev_scale = [&](double tprev) {
        if (tid < 32) {
            double s = 0.0;
            for (int c0 = 0; c0 < G; c0 += 256) {
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const int c = c0 + tid + 32 * u;
                    s += (c < G) ? part_d[c] : 0.0;
                }
            }
            s = warp_sum(s);
            if (tid == 0) s_a2 = -0.5 * tprev * s;
        }
        __syncthreads();
        return s_a2;
    };
    unsigned int bar_target = t.bar_base;
    double tprev = 0.0;
    for (int i = 0; i < t.nb; ++i) {
        const int k = t.j0 + i;
        // ---- phase A: column k of the current matrix on owned rows (the previous column's
        // rank-2 term is formed here from its p and v), partial norm; W of the previous column
        PROF_MARK(0);
        const double a2 = (i > 0) ? prev_scale(tprev) : 0.0;
        if (owner) {
            double ss = 0.0;
            const int r = r_own;
            if (r >= k && r < n) {
                double a = A[(size_t)k * ld + r];
                // all panel columns at once (independent loads; the buffers are zeroed before
                // the first panel, and columns not yet finished get a zero factor)
                double acc = 0.0;
#pragma unroll
                for (int q = 0; q < kPw; ++q) {
                    const double f = (q + 1 < i) ? 1.0 : 0.0;
                    acc += f * (t.V[(size_t)q * n + r] * t.W[(size_t)q * n + k] +
                                t.W[(size_t)q * n + r] * t.V[(size_t)q * n + k]);
                }
                a -= acc;
                if (i > 0) {
                    const double *Vp = t.V + (size_t)(i - 1) * n;
                    const double vr = Vp[r];
                    const double wr = t.ybuf[r] + a2 * vr;
                    const double wk = t.ybuf[k] + a2 * Vp[k];
                    t.W[(size_t)(i - 1) * n + r] = wr;
                    a -= vr * wk + wr * Vp[k];
                }
                t.acol[r] = a;
                if (r >= k + 2) ss = a * a;
            }
            ss = block_sum(ss, red);
            if (tid == 0) part_n[cta] = ss;
        }
        if (!grid_sync_counted(&t.bar->count, bar_target, t.err, t.wait_limit)) return;
        // ---- phase B: reflector (redundantly in every CTA)
        PROF_MARK(1);
        if (tid < 32) {
            double s = 0.0;
            for (int c0 = 0; c0 < NO; c0 += 128) {
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int c = c0 + tid + 32 * u;
                    s += (c < NO) ? part_n[c] : 0.0;
                }
            }
            s = warp_sum(s);
            if (tid == 0) {
                const double alpha = t.acol[k + 1];
                double beta, tk, sc;
                if (s == 0.0) {
                    tk = 0.0;
                    beta = alpha;
                    sc = 0.0;
                } else {
                    beta = -copysign(sqrt(alpha * alpha + s), alpha);
                    tk = (beta - alpha) / beta;
                    sc = 1.0 / (alpha - beta);
                }
                s_tau = tk;
                s_scal = sc;
                if (cta == 0) {
                    t.d[k] = t.acol[k];
                    t.e[k] = beta;
                    t.tau[k] = tk;
                }
            }
        }
        __syncthreads();
        const double tk = s_tau, scal = s_scal;
        tprev = tk;
        auto vval = [&](int r) -> double {
            if (r <= k || r >= n) return 0.0;
            return (r == k + 1) ? 1.0 : t.acol[r] * scal;
        };
        // ---- phase C: s = A22 v over lower tiles of rows/cols >= k+1
        PROF_MARK(2);
        const int t0 = (k + 1) / TB;
        const int ntr = NT - t0;
        const long long ntiles = (long long)ntr * (ntr + 1) / 2;
        if (tk != 0.0 && t.cache_tiles > 0) {
            // resident tiles: the v segments of all of them are fetched up front (independent
            // loads), then two barriers per tile
            const int nmine = ntiles_s > cta ? (int)((ntiles_s - 1 - cta) / G + 1) : 0;
            constexpr int kPre = 6;
            double prev[kPre];
#pragma unroll
            for (int u = 0; u < kPre; ++u) {
                prev[u] = 0.0;
                if (u < nmine && u < t.cache_tiles) {
                    int cI, cJ;
                    decode_rel(cta + (long long)u * G, t0s, cI, cJ);
                    if (cJ >= t0) prev[u] = (tid < TB) ? vval(cI * TB + tid) : (tid < 2 * TB ? vval(cJ * TB + tid - TB) : 0.0);
                }
            }
#pragma unroll
            for (int u = 0; u < kPre; ++u) {
                if (u < nmine && u < t.cache_tiles) {
                    int cI, cJ;
                    decode_rel(cta + (long long)u * G, t0s, cI, cJ);
                    if (cJ >= t0) {
                        const double *Sc = cache + (size_t)u * TB * TS;
                        if (tid < TB) vI[tid] = prev[u];
                        else if (tid < 2 * TB) vJ[tid - TB] = prev[u];
                        __syncthreads();
                        const int r = tid & 63, g = tid >> 6;
                        double acc = 0.0, acc2 = 0.0;
#pragma unroll
                        for (int q = 0; q < 16; ++q) acc += Sc[(g * 16 + q) * TS + r] * vJ[g * 16 + q];
                        if (cI != cJ) {
#pragma unroll
                            for (int q = 0; q < 16; ++q) acc2 += Sc[r * TS + g * 16 + q] * vI[g * 16 + q];
                        }
                        rsum[g][r] = acc;
                        rsJ[g][r] = acc2;
                        __syncthreads();
                        if (tid < TB)
                            t.P[((size_t)cI * NT + cJ) * TB + tid] = rsum[0][tid] + rsum[1][tid] + rsum[2][tid] + rsum[3][tid];
                        else if (cI != cJ && tid < 2 * TB)
                            t.P[((size_t)cJ * NT + cI) * TB + tid - TB] =
                                rsJ[0][tid - TB] + rsJ[1][tid - TB] + rsJ[2][tid - TB] + rsJ[3][tid - TB];
                    }
                }
            }
            // tiles beyond the preloaded ones (cache overflow: streamed from global memory)
            const int ufirst = (t.cache_tiles < kPre) ? t.cache_tiles : kPre;
            for (int u = ufirst; u < nmine; ++u) {
                int cI, cJ;
                decode_rel(cta + (long long)u * G, t0s, cI, cJ);
                if (cJ < t0) continue;
                const double *Sc;
                if (u < t.cache_tiles) {
                    Sc = cache + (size_t)u * TB * TS;
                } else {
                    __syncthreads();
                    const int r0 = cI * TB, c0 = cJ * TB;
                    for (int q = tid; q < TB * TB; q += kPnThreads) {
                        const int c = q / TB, r = q % TB;
                        const int gr = r0 + r, gc = c0 + c;
                        S[c * TS + r] = (gr < n && gc < n) ? __ldcg(A + (size_t)gc * ld + gr) : 0.0;
                    }
                    if (cI == cJ) {
                        __syncthreads();
                        for (int q = tid; q < TB * TB; q += kPnThreads) {
                            const int c = q / TB, r = q % TB;
                            if (r < c) S[c * TS + r] = S[r * TS + c];
                        }
                    }
                    Sc = S;
                }
                if (tid < TB) vI[tid] = vval(cI * TB + tid);
                else if (tid < 2 * TB) vJ[tid - TB] = vval(cJ * TB + tid - TB);
                __syncthreads();
                const int r = tid & 63, g = tid >> 6;
                double acc = 0.0, acc2 = 0.0;
#pragma unroll
                for (int q = 0; q < 16; ++q) acc += Sc[(g * 16 + q) * TS + r] * vJ[g * 16 + q];
                if (cI != cJ) {
#pragma unroll
                    for (int q = 0; q < 16; ++q) acc2 += Sc[r * TS + g * 16 + q] * vI[g * 16 + q];
                }
                rsum[g][r] = acc;
                rsJ[g][r] = acc2;
                __syncthreads();
                if (tid < TB)
                    t.P[((size_t)cI * NT + cJ) * TB + tid] = rsum[0][tid] + rsum[1][tid] + rsum[2][tid] + rsum[3][tid];
                else if (cI != cJ && tid < 2 * TB)
                    t.P[((size_t)cJ * NT + cI) * TB + tid - TB] =
                        rsJ[0][tid - TB] + rsJ[1][tid - TB] + rsJ[2][tid - TB] + rsJ[3][tid - TB];
            }
        } else if (tk != 0.0 && cta < ntiles) {
            // the next tile (and its two v slices) is loaded into registers while the
            // current one is reduced from shared memory; warp w reads columns w, w+8, ..
            // with one 512-byte coalesced row segment per instruction
            double pre[16];
            double pv_pre = 0.0;
            int I = 0, J = 0;
            auto decode = [&](long long tt, int &Io, int &Jo) {
                int li = (int)((sqrt(8.0 * (double)tt + 1.0) - 1.0) * 0.5);
                while ((long long)li * (li + 1) / 2 > tt) --li;
                while ((long long)(li + 1) * (li + 2) / 2 <= tt) ++li;
                Io = t0 + li;
                Jo = t0 + (int)(tt - (long long)li * (li + 1) / 2);
            };
            auto fetch = [&](int Io, int Jo) {
                const int r0 = Io * TB, c0 = Jo * TB;
                const int rr = r0 + 2 * lane;
#pragma unroll
                for (int m = 0; m < 8; ++m) {
                    const int gc = c0 + warp + 8 * m;
                    const double *src = A + (size_t)gc * ld + rr;
                    if (gc < n && rr + 1 < n) {
                        const double2 x = __ldcg(reinterpret_cast<const double2 *>(src));
                        pre[2 * m] = x.x;
                        pre[2 * m + 1] = x.y;
                    } else {
                        pre[2 * m] = (gc < n && rr < n) ? src[0] : 0.0;
                        pre[2 * m + 1] = 0.0;
                    }
                }
                pv_pre = (tid < TB) ? vval(r0 + tid) : (tid < 2 * TB ? vval(c0 + tid - TB) : 0.0);
            };
            decode(cta, I, J);
            fetch(I, J);
            for (long long tt = cta; tt < ntiles; tt += G) {
                const int cI = I, cJ = J;
#pragma unroll
                for (int m = 0; m < 8; ++m) {
                    S[(warp + 8 * m) * TS + 2 * lane] = pre[2 * m];
                    S[(warp + 8 * m) * TS + 2 * lane + 1] = pre[2 * m + 1];
                }
                if (tid < TB) vI[tid] = pv_pre;
                else if (tid < 2 * TB) vJ[tid - TB] = pv_pre;
                if (tt + G < ntiles) {
                    decode(tt + G, I, J);
                    fetch(I, J);
                }
                __syncthreads();
                if (cI == cJ) {
                    // mirror the lower triangle into the upper one
                    for (int q = tid; q < TB * TB; q += kPnThreads) {
                        const int c = q / TB, r = q % TB;
                        if (r < c) S[c * TS + r] = S[r * TS + c];
                    }
                    __syncthreads();
                }
                const int r = tid & 63, g = tid >> 6;
                {   // row products y_I[r] = sum_c S[c][r] vJ[c]
                    double acc = 0.0;
#pragma unroll
                    for (int u = 0; u < 16; ++u) acc += S[(g * 16 + u) * TS + r] * vJ[g * 16 + u];
                    rsum[g][r] = acc;
                }
                double acc2 = 0.0;
                if (cI != cJ) {  // column products y_J[c] = sum_r S[c][r] vI[r]
#pragma unroll
                    for (int u = 0; u < 16; ++u) acc2 += S[r * TS + g * 16 + u] * vI[g * 16 + u];
                }
                __syncthreads();
                if (tid < TB)
                    t.P[((size_t)cI * NT + cJ) * TB + tid] = rsum[0][tid] + rsum[1][tid] + rsum[2][tid] + rsum[3][tid];
                __syncthreads();
                if (cI != cJ) {
                    rsum[g][r] = acc2;
                    __syncthreads();
                    if (tid < TB)
                        t.P[((size_t)cJ * NT + cI) * TB + tid] = rsum[0][tid] + rsum[1][tid] + rsum[2][tid] + rsum[3][tid];
                    __syncthreads();
                }
            }
        }
        // owners: store v (panel column i and reflector storage)
        if (owner) {
            const int r = r_own;
            if (r > k && r < n) {
                const double v = vval(r);
                t.V[(size_t)i * n + r] = v;
                if (r >= k + 2) A[(size_t)k * ld + r] = v;
            }
        }
        // partial V^T v, W^T v: one warp per (panel column, 256-row chunk), over all CTAs
        {
            const int nw = G * (kPnThreads / 32);
            for (int it = cta * (kPnThreads / 32) + warp; it < 2 * i * NO; it += nw) {
                const int q = it / NO, c = it - q * NO;
                const double *x = (q < i) ? t.V + (size_t)q * n : t.W + (size_t)(q - i) * n;
                const int rb = c * kChunk;
                double s = 0.0;
#pragma unroll
                for (int m = 0; m < kChunk / 32; ++m) {
                    const int rr = rb + lane + 32 * m;
                    const int rc = rr < n ? rr : n - 1;
                    const double xv = x[rc], av = t.acol[rc];
                    const double vv = (rr <= k || rr >= n) ? 0.0 : ((rr == k + 1) ? 1.0 : av * scal);
                    s += xv * vv;
                }
                s = warp_sum(s);
                if (lane == 0) part_q[(size_t)c * 2 * nbmax + ((q < i) ? q : nbmax + (q - i))] = s;
            }
        }
        if (!grid_sync_counted(&t.bar->count, bar_target, t.err, t.wait_limit)) return;
        // ---- phase D (all CTAs, eight lanes per row): y_r = sum of the partial products of
        // row r - V (W^T v) - W (V^T v); p = tau y; partial p.v per CTA
        PROF_MARK(3);
        {   // s_corr[q] = (V^T v)_q, s_corr[kPw + q] = (W^T v)_q, zero for q >= i; four
            // threads per value sum interleaved partials
            const int qq = tid & (2 * kPw - 1), pt = tid >> 6;
            const int q = qq & (kPw - 1);
            const int off = (qq < kPw) ? q : nbmax + q;
            double s = 0.0;
            if (q < i) {
                for (int c0 = pt; c0 < NO; c0 += 16) {
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const int c = c0 + 4 * u;
                        s += (c < NO) ? part_q[(size_t)c * 2 * nbmax + off] : 0.0;
                    }
                }
            }
            s_red4[pt][qq] = s;
            __syncthreads();
            if (tid < 2 * kPw) s_corr[tid] = s_red4[0][tid] + s_red4[1][tid] + s_red4[2][tid] + s_red4[3][tid];
        }
        __syncthreads();
        {
            double pvl = 0.0;
            const int sub = lane >> 3, sl = lane & 7;
            for (int rb = k + 1 + (cta * (kPnThreads / 32) + warp) * 4; rb < n; rb += G * (kPnThreads / 8)) {
                const int r = rb + sub;
                double y = 0.0;
                if (r < n) {
                    if (tk != 0.0) {
                        const double *Pr = t.P + ((size_t)(r / TB) * NT) * TB + (r % TB);
                        for (int c0 = t0; c0 < NT; c0 += 32) {
#pragma unroll
                            for (int u = 0; u < 4; ++u) {
                                const int c = c0 + sl + 8 * u;
                                y += (c < NT) ? Pr[(size_t)c * TB] : 0.0;
                            }
                        }
                    }
#pragma unroll
                    for (int u = 0; u < kPw / 8; ++u) {
                        const int q = sl + 8 * u;
                        y -= t.V[(size_t)q * n + r] * s_corr[kPw + q] + t.W[(size_t)q * n + r] * s_corr[q];
                    }
                }
                y += __shfl_xor_sync(0xffffffffu, y, 4);
                y += __shfl_xor_sync(0xffffffffu, y, 2);
                y += __shfl_xor_sync(0xffffffffu, y, 1);
                if (r < n && sl == 0) {
                    const double p = tk * y;
                    t.ybuf[r] = p;
                    pvl += p * vval(r);
                }
            }
            pvl = block_sum(pvl, red);
            if (tid == 0) part_d[cta] = pvl;
        }
        if (!grid_sync_counted(&t.bar->count, bar_target, t.err, t.wait_limit)) return;
    }
    // w of the panel's last column (the kernel boundary orders it before the trailing update)
    PROF_MARK(4);
    {
        const int ip = t.nb - 1, kp = t.j0 + ip;
        const double a2 = prev_scale(tprev);
        if (owner) {
            const int r = r_own;
            if (r > kp && r < n) t.W[(size_t)ip * n + r] = t.ybuf[r] + a2 * t.V[(size_t)ip * n + r];
        }
    }
    PROF_MARK(5);
}

// Trailing update A[j1:, j1:] (lower) -= V W^T + W V^T with DMMA, K = 2 nb.
__device__ __forceinline__ void dmma884d(double &c0, double &c1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

__global__ void __launch_bounds__(128) syr2k_lower_kernel(double *A, long long ld, int n, int j1, const double *V,
                                                          const double *W, int nb) {
    const long long tt = blockIdx.x;
    int li = (int)((sqrt(8.0 * (double)tt + 1.0) - 1.0) * 0.5);
    while ((long long)li * (li + 1) / 2 > tt) --li;
    while ((long long)(li + 1) * (li + 2) / 2 <= tt) ++li;
    const int lj = (int)(tt - (long long)li * (li + 1) / 2);
    const int i0 = j1 + li * 64, jj0 = j1 + lj * 64;
    __shared__ double Xs[64][20];
    __shared__ double Ys[64][20];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    double acc[4][4][2];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
    const int K = 2 * nb;
    for (int k0 = 0; k0 < K; k0 += 16) {
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int e = tid + q * 128;
            const int kk = e / 64, m = e % 64;
            const int gk = k0 + kk;
            double x = 0.0, y = 0.0;
            if (gk < K) {
                const int gi = i0 + m, gj = jj0 + m;
                const double *Xc = (gk < nb) ? V + (size_t)gk * n : W + (size_t)(gk - nb) * n;
                const double *Yc = (gk < nb) ? W + (size_t)gk * n : V + (size_t)(gk - nb) * n;
                if (gi < n) x = Xc[gi];
                if (gj < n) y = Yc[gj];
            }
            Xs[m][kk] = x;
            Ys[m][kk] = y;
        }
        __syncthreads();
        const int r = lane >> 2, c = lane & 3;
#pragma unroll
        for (int kk = 0; kk < 16; kk += 4) {
            double af[4], bf[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) af[q] = Xs[wm + q * 8 + r][kk + c];
#pragma unroll
            for (int q = 0; q < 4; ++q) bf[q] = Ys[wn + q * 8 + r][kk + c];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) dmma884d(acc[a][b][0], acc[a][b][1], af[a], bf[b]);
        }
        __syncthreads();
    }
    const int r = lane >> 2, c2 = (lane & 3) * 2;
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int i = i0 + wm + a * 8 + r, j = jj0 + wn + b * 8 + c2 + h;
                if (i < n && j < n && i >= j) A[(size_t)j * ld + i] -= acc[a][b][h];
            }
}

__global__ void dense_finish_kernel(const double *A, long long ld, int n, double *d, double *e, double *tau) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    if (n == 1) {
        d[0] = A[0];
        e[0] = 0.0;
        tau[0] = 0.0;
        return;
    }
    d[n - 2] = A[(size_t)(n - 2) * ld + (n - 2)];
    d[n - 1] = A[(size_t)(n - 1) * ld + (n - 1)];
    e[n - 2] = A[(size_t)(n - 2) * ld + (n - 1)];
    e[n - 1] = 0.0;
    tau[n - 2] = 0.0;
    tau[n - 1] = 0.0;
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
// Eigenvalues closer than ortol_rel ||T|| form a cluster whose vectors are computed in turn
// and orthogonalised against each other; apart, inverse iteration's own accuracy
// (eps ||T|| / gap) is their orthogonality.
__global__ void clusters_kernel(const double *w, int nev, const double *info, double ortol_rel, int *cstart, int *ncl) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double ortol = ortol_rel * info[3];
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
        invit_cluster(d, e, n, w, cstart[c], cstart[c + 1], info[3], fac, T, t, X, nev, nullptr);
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
                                     double *Z, long long ldz, int nev) {
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int c0 = gw * kBtCols;
    if (c0 >= nev) return;
    const int nc = min(kBtCols, nev - c0);
    for (int k = n - 3; k >= 0; --k) {
        const double tk = tau[k];
        if (tk == 0.0) continue;
        const double *col = A + (size_t)k * lda;
        double s[kBtCols] = {0.0, 0.0, 0.0, 0.0};
        for (int i = k + 1 + lane; i < n; i += 32) {
            const double vi = (i == k + 1) ? 1.0 : col[i];
#pragma unroll
            for (int c = 0; c < kBtCols; ++c)
                if (c < nc) s[c] += vi * Z[(size_t)(c0 + c) * ldz + i];
        }
#pragma unroll
        for (int c = 0; c < kBtCols; ++c) s[c] = warp_sum(s[c]) * tk;
        for (int i = k + 1 + lane; i < n; i += 32) {
            const double vi = (i == k + 1) ? 1.0 : col[i];
#pragma unroll
            for (int c = 0; c < kBtCols; ++c)
                if (c < nc) Z[(size_t)(c0 + c) * ldz + i] -= s[c] * vi;
        }
    }
}

// ---- eigenvectors of T by inverse iteration with the factors in shared memory
// One warp per cluster (1 warp per CTA). The recurrences (LU with partial pivoting of
// T - lambda I, forward and backward solves) run on lane 0 from shared memory; scaling,
// Gram-Schmidt inside the cluster and normalisation use the whole warp. Same steps as
// invit_cluster (dstein manner), written straight into column-major Z.
__global__ void __launch_bounds__(32) invit_smem_kernel(const double *d, const double *e, int n, const double *w,
                                                        const int *cstart, const int *ncl, const double *info,
                                                        double *Z, long long ldz) {
    extern __shared__ double sm[];
    double *D = sm, *E1 = D + n, *E2 = E1 + n, *Lm = E2 + n, *x = Lm + n;
    unsigned char *P = reinterpret_cast<unsigned char *>(x + n);
    const int lane = threadIdx.x;
    const int nc = *ncl;
    const double onenrm = info[3];
    const double eps = DBL_EPSILON, tiny = eps * onenrm, pertol = 10.0 * eps * onenrm;
    for (int c = blockIdx.x; c < nc; c += gridDim.x) {
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
            // the solves below multiply by the pivots' reciprocals (one division per pivot here
            // instead of one per pivot and iteration on the sequential path)
            const double dlast = D[n - 1];
            __syncwarp();
            for (int i = lane; i < n; i += 32) D[i] = 1.0 / D[i];
            for (int i = lane; i < n; i += 32) {
                const unsigned h = hash32((unsigned)(i * 2654435761u) ^ (unsigned)(j * 40503u + 17u));
                x[i] = ((double)(h & 0xffffff) / 8388608.0) - 1.0;
            }
            __syncwarp();
            for (int it = 0; it < 4; ++it) {
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
                    const double *zc = Z + (size_t)jj * ldz;
                    double dot = 0.0;
                    for (int i = lane; i < n; i += 32) dot += x[i] * zc[i];
                    dot = warp_sum(dot);
                    for (int i = lane; i < n; i += 32) x[i] -= dot * zc[i];
                }
                double nrm = 0.0;
                for (int i = lane; i < n; i += 32) nrm += x[i] * x[i];
                nrm = sqrt(warp_sum(nrm));
                const double inv = (nrm > 0.0) ? 1.0 / nrm : 0.0;
                for (int i = lane; i < n; i += 32) x[i] *= inv;
                __syncwarp();
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
            double *zc = Z + (size_t)j * ldz;
            for (int i = lane; i < n; i += 32) zc[i] = sg * x[i];
            __syncwarp();
        }
    }
}

// ---- blocked back-transformation Z <- H_0 H_1 ... H_{n-3} Z (compact WY, as dormtr)
// V panel (rows p0..n-1, nbk columns): column c is reflector p0+c, zero above row p0+c+1,
// one at row p0+c+1, A[r, p0+c] below.
__global__ void build_v_kernel(const double *A, long long lda, int n, int p0, int nbk, double *V, long long ldv) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int R = n - p0;
    if (t >= (long long)R * nbk) return;
    const int c = (int)(t / R), i = (int)(t % R);
    const int r = p0 + i, top = p0 + c + 1;
    V[(size_t)c * ldv + i] = (r < top) ? 0.0 : (r == top ? 1.0 : A[(size_t)(p0 + c) * lda + r]);
}

// Tm (upper, ld 32) of the block reflector I - V Tm V^T from S = V^T V (ld 32) and tau (dlarft,
// forward, columnwise).
__global__ void larft_kernel(const double *S, const double *tau, int nbk, double *Tm) {
    __shared__ double t[32][33], sv[32][33], ts[32];
    const int r = threadIdx.x;
    for (int c = 0; c < 32; ++c) {
        t[r][c] = 0.0;
        sv[c][r] = (r < nbk && c < nbk) ? S[c * 32 + r] : 0.0;  // sv[i][c] = S(c, i)
    }
    ts[r] = (r < nbk) ? tau[r] : 0.0;
    __syncwarp();
    for (int i = 0; i < nbk; ++i) {
        const double ti = ts[i];
        if (r < i) {
            double s = 0.0;
            for (int c = r; c < i; ++c) s += t[r][c] * sv[i][c];
            t[r][i] = -ti * s;
        } else if (r == i) {
            t[i][i] = ti;
        }
        __syncwarp();
    }
    for (int c = 0; c < 32; ++c) Tm[c * 32 + r] = t[r][c];
}

}  // namespace

size_t dense_bt_work_doubles(int n, int nev) {
    const long long ldv = (n + 7) / 8 * 8;
    return (size_t)ldv * 32 + 2 * 32 * 32 + 2 * (size_t)32 * nev + (size_t)64 * 32 * nev + 64;
}

cudaError_t launch_dense_backtransform(const double *A, long long lda, int n, const double *tau, double *Z,
                                       long long ldz, int nev, double *work, cudaStream_t st) {
    if (n < 3 || nev <= 0) return cudaSuccess;
    if (ldz & 1) return cudaErrorInvalidValue;
    const long long ldv = (n + 7) / 8 * 8;
    double *V = work, *S = V + ldv * 32, *Tm = S + 32 * 32, *W = Tm + 32 * 32, *W2 = W + (size_t)32 * nev;
    double *sk = W2 + (size_t)32 * nev;
    cudaError_t e;
    const int nref = n - 2;
    const int npan = (nref + 31) / 32;
    for (int q = npan - 1; q >= 0; --q) {
        const int p0 = q * 32, nbk = std::min(32, nref - p0), R = n - p0;
        DVR3D_COUNT_LAUNCH(1);
        build_v_kernel<<<(unsigned)(((long long)R * nbk + 255) / 256), 256, 0, st>>>(A, lda, n, p0, nbk, V, ldv);
        GemmOp g;  // S = V^T V
        g.M = nbk;
        g.N = nbk;
        g.K = R;
        g.A = V;
        g.lda = ldv;
        g.ta = true;
        g.B = V;
        g.ldb = ldv;
        g.C = S;
        g.ldc = 32;
        g.splitk = std::max(1, std::min(64, (R + 15) / 16 / 8));
        g.work = sk;
        if ((e = launch_gemm(g, st)) != cudaSuccess) return e;
        DVR3D_COUNT_LAUNCH(1);
        larft_kernel<<<1, 32, 0, st>>>(S, tau + p0, nbk, Tm);
        GemmOp a;  // W = V^T Z[p0:, :]
        a.M = nbk;
        a.N = nev;
        a.K = R;
        a.A = V;
        a.lda = ldv;
        a.ta = true;
        a.B = Z + p0;
        a.ldb = ldz;
        a.C = W;
        a.ldc = 32;
        const int tiles = (nev + 63) / 64;
        a.splitk = std::max(1, std::min(64, std::min((600 + tiles - 1) / tiles, (R + 15) / 16)));
        a.work = sk;
        if ((e = launch_gemm(a, st)) != cudaSuccess) return e;
        GemmOp b;  // W2 = Tm W
        b.M = nbk;
        b.N = nev;
        b.K = nbk;
        b.A = Tm;
        b.lda = 32;
        b.B = W;
        b.ldb = 32;
        b.C = W2;
        b.ldc = 32;
        if ((e = launch_gemm(b, st)) != cudaSuccess) return e;
        GemmOp c;  // Z[p0:, :] -= V W2
        c.M = R;
        c.N = nev;
        c.K = nbk;
        c.alpha = -1.0;
        c.beta = 1.0;
        c.A = V;
        c.lda = ldv;
        c.B = W2;
        c.ldb = 32;
        c.C = Z + p0;
        c.ldc = ldz;
        if ((e = launch_gemm(c, st)) != cudaSuccess) return e;
    }
    return cudaGetLastError();
}

int dense_tridiag_grid(int device) {
    int nsm = 0, per = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
    cudaFuncSetAttribute(dense_panel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, dense_panel_kernel, kPnThreads, (size_t)TB * TS * sizeof(double));
    if (per < 1) per = 1;
    return nsm * std::min(per, 3);
}

int dense_panel_width() { return kPw; }

int dense_resident_plan(int device, int n, int *grid) {
    // one CTA per SM with as many 64 x 64 tiles as fit next to the scratch tile; used while
    // most of the lower tiles of the matrix fit on chip (about n <= 2900 on B200)
    int nsm = 0, smem_optin = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
    cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    const size_t tile = (size_t)TB * TS * sizeof(double);
    const int slots = (int)((smem_optin - 8 * 1024) / tile) - 1;  // static shared memory kept aside
    if (slots < 1) return 0;
    const long long NT = (n + TB - 1) / TB, ntiles = NT * (NT + 1) / 2;
    if (ntiles > (long long)nsm * slots * 5 / 4) return 0;
    cudaError_t e = cudaFuncSetAttribute(dense_panel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)(((size_t)slots + 1) * tile));
    if (e != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    int per = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, dense_panel_kernel, kPnThreads, ((size_t)slots + 1) * tile);
    if (per < 1) return 0;
    *grid = nsm;
    return slots;
}

cudaError_t launch_dense_tridiag(DenseTri &t, int grid, cudaStream_t st) {
    const int n = t.n;
    const int nb = t.nbmax;
    if (nb != kPw) return cudaErrorInvalidValue;
    int npanel = 0;
    t.bar_base = 0;
    for (int j0 = 0; j0 + 2 < n; j0 += nb) {
        t.j0 = j0;
        t.nb = std::min(nb, n - 2 - j0);
        void *args[] = {&t};
        if (t.ev && 2 * npanel + 1 < t.nev) cudaEventRecord(t.ev[2 * npanel], st);
        DVR3D_COUNT_LAUNCH(1);
        const size_t smem = ((size_t)t.cache_tiles + 1) * TB * TS * sizeof(double);
        cudaError_t e = cudaLaunchCooperativeKernel((void *)dense_panel_kernel, dim3(grid), dim3(kPnThreads), args, smem, st);
        if (t.ev && 2 * npanel + 1 < t.nev) cudaEventRecord(t.ev[2 * npanel + 1], st);
        ++npanel;
        t.bar_base += 3u * (unsigned)t.nb * (unsigned)grid;  // three barriers per column
        if (e != cudaSuccess) return e;
        const int j1 = j0 + t.nb;
        if (j1 < n) {
            const long long nt = (n - j1 + 63) / 64;
            DVR3D_COUNT_LAUNCH(1);
            syr2k_lower_kernel<<<(unsigned)(nt * (nt + 1) / 2), 128, 0, st>>>(t.A, t.lda, n, j1, t.V, t.W, t.nb);
            e = cudaGetLastError();
            if (e != cudaSuccess) return e;
        }
    }
    DVR3D_COUNT_LAUNCH(1);
    dense_finish_kernel<<<1, 32, 0, st>>>(t.A, t.lda, n, t.d, t.e, t.tau);
    t.npanel = npanel;
    return cudaGetLastError();
}

void launch_dense_eigvals(const double *d, const double *e, int n, int nev, double *e2, double *info,
                          double *w, cudaStream_t st) {
    DVR3D_COUNT_LAUNCH(2);
    tri_bounds_kernel<<<1, 256, 0, st>>>(d, e, n, e2, info);
    const int warps_per_block = 4;
    multisect_kernel<<<(nev + warps_per_block - 1) / warps_per_block, 32 * warps_per_block, 0, st>>>(
        d, e2, n, nev, info, w);
}

void launch_tridiag_eigvecs(const double *d, const double *e, int n, const double *w, int nev, const double *info,
                            int *cstart, int *ncl, double *fac, int T, double *X, double *Z, long long ldz,
                            double ortol_rel, cudaStream_t st) {
    DVR3D_COUNT_LAUNCH(1);
    clusters_kernel<<<1, 32, 0, st>>>(w, nev, info, ortol_rel, cstart, ncl);
    const size_t smem = invit_smem_bytes(n);
    if (smem <= (size_t)kInvitSmemMax) {
        int dev = 0;
        cudaGetDevice(&dev);
        static bool attr[kMaxAttrDevices] = {};
        if (dev < 0 || dev >= kMaxAttrDevices || !attr[dev]) {
            cudaFuncSetAttribute(invit_smem_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kInvitSmemMax);
            if (dev >= 0 && dev < kMaxAttrDevices) attr[dev] = true;
        }
        DVR3D_COUNT_LAUNCH(1);
        invit_smem_kernel<<<nev, 32, smem, st>>>(d, e, n, w, cstart, ncl, info, Z, ldz);
    } else {
        DVR3D_COUNT_LAUNCH(2);
        invit_dense_kernel<<<(T + 63) / 64, 64, 0, st>>>(d, e, n, w, nev, cstart, ncl, info, fac, T, X);
        const long long tot = (long long)n * nev;
        untangle_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(X, n, nev, Z, ldz);
    }
}

void launch_dense_eigvecs(const double *A, long long lda, int n, const double *d, const double *e,
                          const double *tau, const double *w, int nev,
                          const double *info, int *cstart, int *ncl, double *fac, int T, double *X,
                          double *Z, long long ldz, double *bt_work, cudaStream_t st) {
    launch_tridiag_eigvecs(d, e, n, w, nev, info, cstart, ncl, fac, T, X, Z, ldz, 1.0e-6, st);
    if (bt_work && !(ldz & 1)) {
        launch_dense_backtransform(A, lda, n, tau, Z, ldz, nev, bt_work, st);
    } else {
        DVR3D_COUNT_LAUNCH(1);
        const int nwarps = (nev + kBtCols - 1) / kBtCols;
        backtransform_kernel<<<(nwarps + 3) / 4, 128, 0, st>>>(A, lda, n, tau, Z, ldz, nev);
    }
}

size_t invit_smem_bytes(int n) { return (size_t)n * (5 * sizeof(double) + 1) + 16; }

}  // namespace dvr3d
