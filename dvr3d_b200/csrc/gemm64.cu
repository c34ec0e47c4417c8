// gemm64.cu -- FP64 tensor-core (DMMA, mma.sync m8n8k4 .f64) kernels.
//
// (1) assemble_h3: the contracted 3D Hamiltonian
//        H3[i,j] = T[g(i), g(j)] * sum_p Vt[p,i] Vt[p,j]  +  delta_ij e2[i]
//     which is what bloc3d/blc2d2/vecmul (:3455-3595, Radau) and mkham3/loadh
//     (:2301-2609, Jacobi) compute block pair by block pair; here it is one block-scaled
//     SYRK over lower 64x64 tiles, mirrored into full symmetric storage.
// (2) dgemm: C = alpha op(A) op(B) + beta C (column-major), used by the eigenvector
//     back-transforms, residuals and the Davidson solver.
#include <cuda_runtime.h>

#include "common.cuh"
#include "gemm64.cuh"

namespace dvr3d {

namespace {

constexpr int BM = 64, BN = 64, BK = 16, PAD = 4, LDS = BK + PAD;
constexpr int kThreads = 128;  // 4 warps, 2 x 2, each 32 x 32

__device__ __forceinline__ void dmma884(double &c0, double &c1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

// Warp computes a 32x32 tile from As[m][k], Bs[n][k] (k contiguous), BK deep.
__device__ __forceinline__ void warp_tile_mma(const double (*As)[LDS], const double (*Bs)[LDS],
                                              int wm, int wn, int lane, double acc[4][4][2]) {
    const int r = lane >> 2, c = lane & 3;
#pragma unroll
    for (int kk = 0; kk < BK; kk += 4) {
        double af[4], bf[4];
#pragma unroll
        for (int t = 0; t < 4; ++t) af[t] = As[wm + t * 8 + r][kk + c];
#pragma unroll
        for (int t = 0; t < 4; ++t) bf[t] = Bs[wn + t * 8 + r][kk + c];
#pragma unroll
        for (int ti = 0; ti < 4; ++ti)
#pragma unroll
            for (int tj = 0; tj < 4; ++tj) dmma884(acc[ti][tj][0], acc[ti][tj][1], af[ti], bf[tj]);
    }
}

// ---------------------------------------------------------------- H3 assembly
__global__ void __launch_bounds__(kThreads) assemble_h3_kernel(AsmParams p) {
    // lower tile pair (ti >= tj) from the linear block index
    const long long t = blockIdx.x;
    int ti = (int)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
    while ((long long)ti * (ti + 1) / 2 > t) --ti;
    while ((long long)(ti + 1) * (ti + 2) / 2 <= t) ++ti;
    const int tj = (int)(t - (long long)ti * (ti + 1) / 2);
    const int i0 = ti * BM, j0 = tj * BN;
    __shared__ __align__(16) double As[2][BM][LDS];
    __shared__ __align__(16) double Bs[2][BN][LDS];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    double acc[4][4][2];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
    const double *Vt = p.Vt;
    const long long ldv = p.ldv;
    // each thread copies 8 doubles of A and 8 of B per stage with 16-byte cp.async
    auto load_stage = [&](int st, int k0) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int e = tid + q * kThreads;  // 0..511 pairs
            const int row = e >> 3, kp = (e & 7) * 2;
            const double *ga = Vt + (size_t)(i0 + row) * ldv + k0 + kp;
            const double *gb = Vt + (size_t)(j0 + row) * ldv + k0 + kp;
            unsigned sa = (unsigned)__cvta_generic_to_shared(&As[st][row][kp]);
            unsigned sb = (unsigned)__cvta_generic_to_shared(&Bs[st][row][kp]);
            asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(ga));
            asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(sb), "l"(gb));
        }
        asm volatile("cp.async.commit_group;\n" ::);
    };
    const int nk = (int)(ldv / BK);
    load_stage(0, 0);
    for (int kt = 0; kt < nk; ++kt) {
        const int st = kt & 1;
        if (kt + 1 < nk) {
            load_stage(st ^ 1, (kt + 1) * BK);
            asm volatile("cp.async.wait_group 1;\n" ::);
        } else {
            asm volatile("cp.async.wait_group 0;\n" ::);
        }
        __syncthreads();
        warp_tile_mma(As[st], Bs[st], wm, wn, lane, acc);
        __syncthreads();
    }
    // epilogue: block scale, diagonal, full symmetric store
    const int r = lane >> 2, c2 = (lane & 3) * 2;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
#pragma unroll
        for (int b = 0; b < 4; ++b) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int i = i0 + wm + a * 8 + r;
                const int j = j0 + wn + b * 8 + c2 + h;
                if (i >= p.n || j >= p.n) continue;
                if (ti == tj && j > i) continue;  // diagonal tile: lower half only
                double v = acc[a][b][h] * p.T[(size_t)p.g[j] * p.ldt + p.g[i]];
                if (i == j) v += p.e2[i];
                p.H[(size_t)j * p.ldh + i] = v;
                p.H[(size_t)i * p.ldh + j] = v;
            }
        }
    }
}

// ---------------------------------------------------------------- general DGEMM
// op(A) is M x K, op(B) is K x N, column-major storage.
template <bool TA, bool TB>
__global__ void __launch_bounds__(kThreads) dgemm_kernel(int M, int N, int K, double alpha,
                                                          const double *__restrict__ A, long long lda,
                                                          const double *__restrict__ B, long long ldb,
                                                          double beta, double *C, long long ldc) {
    __shared__ __align__(16) double As[BM][LDS];
    __shared__ __align__(16) double Bs[BN][LDS];
    const int i0 = blockIdx.y * BM, j0 = blockIdx.x * BN;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    double acc[4][4][2];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
    for (int k0 = 0; k0 < K; k0 += BK) {
        // A tile: As[m][k] = opA(i0+m, k0+k)
#pragma unroll
        for (int q = 0; q < (BM * BK) / kThreads; ++q) {
            const int e = tid + q * kThreads;
            int m, k;
            if (TA) {  // op(A)(i,k) = A[i*lda + k]: contiguous in k
                m = e / BK;
                k = e % BK;
            } else {   // A[k*lda + i]: contiguous in i
                k = e / BM;
                m = e % BM;
            }
            const int gi = i0 + m, gk = k0 + k;
            double v = 0.0;
            if (gi < M && gk < K) v = TA ? A[(size_t)gi * lda + gk] : A[(size_t)gk * lda + gi];
            As[m][k] = v;
        }
#pragma unroll
        for (int q = 0; q < (BN * BK) / kThreads; ++q) {
            const int e = tid + q * kThreads;
            int n, k;
            if (TB) {  // op(B)(k,j) = B[k*ldb + j]: contiguous in j
                k = e / BN;
                n = e % BN;
            } else {   // B[j*ldb + k]: contiguous in k
                n = e / BK;
                k = e % BK;
            }
            const int gj = j0 + n, gk = k0 + k;
            double v = 0.0;
            if (gj < N && gk < K) v = TB ? B[(size_t)gk * ldb + gj] : B[(size_t)gj * ldb + gk];
            Bs[n][k] = v;
        }
        __syncthreads();
        warp_tile_mma(As, Bs, wm, wn, lane, acc);
        __syncthreads();
    }
    const int r = lane >> 2, c2 = (lane & 3) * 2;
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int i = i0 + wm + a * 8 + r, j = j0 + wn + b * 8 + c2 + h;
                if (i < M && j < N) {
                    double *cp = C + (size_t)j * ldc + i;
                    const double old = (beta != 0.0) ? *cp : 0.0;
                    *cp = alpha * acc[a][b][h] + beta * old;
                }
            }
}

// ---------------------------------------------------------------- grouped DGEMM
template <bool TA>
__global__ void __launch_bounds__(kThreads) grouped_dgemm_kernel(GroupedGemm gg) {
    const int t = blockIdx.x;
    int g = 0;
    while (g + 1 < gg.ngroups && gg.tile_start[g + 1] <= t) ++g;
    const int M = gg.M[g], K = gg.K[g], N = gg.N;
    const int tm = (M + BM - 1) / BM;
    const int local = t - gg.tile_start[g];
    const int i0 = (local % tm) * BM, j0 = (local / tm) * BN;
    const double *A = gg.A + gg.aoff[g];
    const double *B = gg.B + gg.boff[g];
    double *C = gg.C + gg.coff[g];
    const long long lda = gg.lda, ldb = gg.ldb, ldc = gg.ldc;
    __shared__ __align__(16) double As[BM][LDS];
    __shared__ __align__(16) double Bs[BN][LDS];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    double acc[4][4][2];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
    for (int k0 = 0; k0 < K; k0 += BK) {
#pragma unroll
        for (int q = 0; q < (BM * BK) / kThreads; ++q) {
            const int e = tid + q * kThreads;
            int m, k;
            if (TA) {
                m = e / BK;
                k = e % BK;
            } else {
                k = e / BM;
                m = e % BM;
            }
            const int gi = i0 + m, gk = k0 + k;
            double v = 0.0;
            if (gi < M && gk < K) v = TA ? A[(size_t)gi * lda + gk] : A[(size_t)gk * lda + gi];
            As[m][k] = v;
        }
#pragma unroll
        for (int q = 0; q < (BN * BK) / kThreads; ++q) {
            const int e = tid + q * kThreads;
            const int n = e / BK, k = e % BK;
            const int gj = j0 + n, gk = k0 + k;
            Bs[n][k] = (gj < N && gk < K) ? B[(size_t)gj * ldb + gk] : 0.0;
        }
        __syncthreads();
        warp_tile_mma(As, Bs, wm, wn, lane, acc);
        __syncthreads();
    }
    const int r = lane >> 2, c2 = (lane & 3) * 2;
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int i = i0 + wm + a * 8 + r, j = j0 + wn + b * 8 + c2 + h;
                if (i < M && j < N) {
                    double *cp = C + (size_t)j * ldc + i;
                    const double old = (gg.beta != 0.0) ? *cp : 0.0;
                    *cp = gg.alpha * acc[a][b][h] + gg.beta * old;
                }
            }
}

}  // namespace

void launch_grouped_dgemm(const GroupedGemm &g, bool transA, int total_tiles, cudaStream_t st) {
    if (total_tiles <= 0) return;
    DVR3D_COUNT_LAUNCH(1);
    if (transA) grouped_dgemm_kernel<true><<<total_tiles, kThreads, 0, st>>>(g);
    else grouped_dgemm_kernel<false><<<total_tiles, kThreads, 0, st>>>(g);
}

void launch_assemble_h3(const AsmParams &p, cudaStream_t st) {
    const long long tiles = (long long)((p.n + BM - 1) / BM);
    const long long nblk = tiles * (tiles + 1) / 2;
    if (nblk == 0) return;
    DVR3D_COUNT_LAUNCH(1);
    assemble_h3_kernel<<<(unsigned)nblk, kThreads, 0, st>>>(p);
}

void launch_dgemm(bool ta, bool tb, int M, int N, int K, double alpha, const double *A, long long lda,
                  const double *B, long long ldb, double beta, double *C, long long ldc, cudaStream_t st) {
    if (M <= 0 || N <= 0) return;
    dim3 grid((N + BN - 1) / BN, (M + BM - 1) / BM);
    DVR3D_COUNT_LAUNCH(1);
    if (!ta && !tb) dgemm_kernel<false, false><<<grid, kThreads, 0, st>>>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
    else if (ta && !tb) dgemm_kernel<true, false><<<grid, kThreads, 0, st>>>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
    else if (!ta && tb) dgemm_kernel<false, true><<<grid, kThreads, 0, st>>>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
    else dgemm_kernel<true, true><<<grid, kThreads, 0, st>>>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
}

}  // namespace dvr3d
