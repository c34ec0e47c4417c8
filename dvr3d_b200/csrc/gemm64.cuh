// gemm64.cuh -- FP64 tensor-core kernels (assembly SYRK, general DGEMM).
#pragma once

#include <cuda_runtime.h>

namespace dvr3d {

struct AsmParams {
    const double *Vt;   // P x ncol_alloc, column-major, ldv (multiple of 16, zero padded)
    long long ldv;
    int n;              // N: number of basis functions (columns used)
    const int *g;       // [N] block (angle / last-coordinate point) of each column
    const double *T;    // block coupling matrix T[g, g'] (ldt), e.g. the L matrix
    int ldt;
    const double *e2;   // [N] diagonal addition (2D eigenvalues)
    double *H;          // N x N output, full symmetric storage, ldh
    long long ldh;
};

void launch_assemble_h3(const AsmParams &p, cudaStream_t st);

// C = alpha op(A) op(B) + beta C; op(A) is M x K, op(B) is K x N; column-major.
void launch_dgemm(bool ta, bool tb, int M, int N, int K, double alpha, const double *A, long long lda,
                  const double *B, long long ldb, double beta, double *C, long long ldc, cudaStream_t st);

// Grouped GEMM, one launch for many independent problems with their own M and K:
//   C_g (M_g x N) = alpha * op(A_g) (M_g x K_g) * B_g (K_g x N) + beta * C_g
// op(A) = A (column-major, lda) or A^T (A stored K_g x M_g column-major, lda);
// B_g, C_g column-major with ldb, ldc. All pointers device; per-group arrays device.
struct GroupedGemm {
    int ngroups;
    const int *tile_start;     // [ngroups+1] prefix of 64x64 output tiles
    const int *M, *K;          // [ngroups]
    int N;
    const double *A;
    const long long *aoff;
    long long lda;
    const double *B;
    const long long *boff;
    long long ldb;
    double *C;
    const long long *coff;
    long long ldc;
    double alpha, beta;
};

void launch_grouped_dgemm(const GroupedGemm &g, bool transA, int total_tiles, cudaStream_t st);

// Pipelined DMMA GEMM: C (M x N, ldc) = alpha op(A) op(B) + beta C.
//   op(A) is M x K: ta ? A stored K x M (element (i,k) at A[i*lda+k]) : A[k*lda+i]
//   op(B) is K x N: tb ? B stored N x K (element (k,j) at B[k*ldb+j]) : B[j*ldb+k]
//   tri = 1: op(A) lower triangular (only k <= i contributes), 2: upper (only k >= i);
//   tri_b = 1: op(B) lower triangular (only k >= j contributes), 2: upper (only k <= j);
//            the other triangle must hold zeros (only whole k tiles are skipped)
//   lower_out: M == N, only C(i,j) with i >= j is computed and written
//   splitk > 1: K split over that many CTAs per tile; up to 8 slices form a thread-block
//            cluster and sum their partial tiles through distributed shared memory (work
//            unused); more slices need work (gemm_splitk_work(M, N, splitk) doubles) and a
//            second reduction kernel
// A, B 16-byte aligned, lda and ldb even.
struct GemmOp {
    int M = 0, N = 0, K = 0;
    double alpha = 1.0, beta = 0.0;
    const double *A = nullptr;
    long long lda = 0;
    const double *B = nullptr;
    long long ldb = 0;
    double *C = nullptr;
    long long ldc = 0;
    bool ta = false, tb = false;
    int tri = 0;
    int tri_b = 0;
    int lower_out = 0;
    int splitk = 1;
    double *work = nullptr;
};
size_t gemm_splitk_work(int M, int N, int splitk);
cudaError_t launch_gemm(const GemmOp &p, cudaStream_t st);

// Algorithmic flops of one launch_gemm: 2 per multiply-add of a nonzero term (triangular
// operands and a lower-triangle output count only their nonzero / computed part).
double gemm_alg_flops(const GemmOp &p);

// Per-launch timing of launch_gemm, the dominant kernel family of the iterative solves: while
// a log is installed on the calling host thread, each launch_gemm records a CUDA event before
// and after its kernels (events from `ev`, two per launch) and adds its algorithmic flops.
struct GemmLaunchLog {
    cudaEvent_t *ev = nullptr;
    int nev = 0;
    int used = 0;        // events recorded
    int launches = 0;    // launches timed
    int untimed = 0;     // launches after the event pool ran out
    double flops = 0.0;  // algorithmic flops of the timed launches
};
void set_gemm_launch_log(GemmLaunchLog *log);  // nullptr: stop logging
// Sum of the timed launches' durations (ms); synchronises on the last event.
double gemm_launch_log_ms(const GemmLaunchLog &log);

}  // namespace dvr3d
