// eig_dense.cuh -- FP64 eigensolver for the final Hamiltonian (lowest levels).
#pragma once

#include <cuda_runtime.h>

#include "common.cuh"

namespace dvr3d {

struct DenseTri {
    double *A;          // n x n full symmetric (overwritten: reflectors below the subdiagonal)
    long long lda;
    int n;
    double *d, *e, *tau, *scal;   // [n]
    double *vp, *wp, *pbuf;       // [n] pending rank-2 vectors and p
    double *part;                 // [2 * grid] partial sums
    GridBarrier *bar;             // zeroed before launch
    int *err;
};

int dense_tridiag_grid(int device);
cudaError_t launch_dense_tridiag(DenseTri &t, int grid, cudaStream_t st);
// info[0..3] = lower bound, upper bound, pivmin, ||T||
void launch_dense_eigvals(const double *d, const double *e, int n, int nev, double *e2, double *info,
                          double *w, cudaStream_t st);
void launch_dense_eigvecs(const double *A, long long lda, int n, const double *d, const double *e,
                          const double *tau, const double *scal, const double *w, int nev,
                          const double *info, int *cstart, int *ncl, double *fac, int T, double *X,
                          double *Z, long long ldz, cudaStream_t st);

}  // namespace dvr3d
