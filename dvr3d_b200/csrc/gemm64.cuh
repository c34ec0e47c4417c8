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

}  // namespace dvr3d
