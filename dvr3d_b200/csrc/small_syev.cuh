// small_syev.cuh -- shared-memory symmetric eigensolver (n <= 160), one CTA per matrix.
#pragma once

#include <cuda_runtime.h>

namespace dvr3d {

constexpr int kSmallSyevMax = 160;

struct SmallSyev {
    int nmat;
    const int *n;             // [nmat] dimensions (<= 160), device
    const double *A;          // matrices (lower triangle read), column-major
    const long long *aoff;    // [nmat] offsets into A
    const long long *lda;     // [nmat] leading dimensions, or null for lda = n
    double *W;                // eigenvalues, ascending
    const long long *woff;    // [nmat]
    double *Z;                // eigenvectors (n x n, ld n), or null for eigenvalues only
    const long long *zoff;    // [nmat]
    double *work;             // inverse-iteration work, small_syev_work_doubles(n) per matrix
    const long long *workoff; // [nmat]
};

size_t small_syev_smem(int nmax);
long long small_syev_work_doubles(int n);
cudaError_t launch_small_syev(const SmallSyev &p, int nmax, cudaStream_t st);

}  // namespace dvr3d
