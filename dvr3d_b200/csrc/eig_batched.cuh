// eig_batched.cuh -- batched FP64 symmetric eigensolver for many independent blocks.
//
// Replaces the reference's per-block calls diag(ham,maxham,nham,eig) -> LAPACK
// dsyev('V','L') (source/dvr3drjz_segmented.f90:2638-2659) in the 1D (jhmain :1987) and 2D
// (jhmain :2030, nfmain :3077) stages. Only the eigenpairs that the energy cut-off keeps
// are needed downstream, so the solver is split the way dsyevx is:
//   1. Householder tridiagonalisation, one CTA per block (reflectors kept in the block);
//   2. Sturm-count bisection: either the eigenvalues below a cut-off or all of them;
//   3. inverse iteration (with modified Gram-Schmidt inside clusters of close eigenvalues)
//      for the selected eigenvalues only, then back-transformation by the reflectors.
// Every block lives in global memory (L2-resident for the sizes of the 1D/2D stages).
#pragma once

#include <cuda_runtime.h>

namespace dvr3d {

struct BatchDesc {
    int nblk;
    const int *n;            // [nblk] block dimension
    const long long *aoff;   // [nblk] offset of block b in A (column-major, ld = n[b])
    const long long *voff;   // [nblk] offset of block b in the n-length arrays d, e, tau, w
};

// Mirror the lower triangle of every block into its upper triangle (the reference's
// dsyev('V','L') reads only the lower triangle; the kernels here use full storage).
void launch_symmetrize_lower(const BatchDesc &bd, double *A, int nmax, cudaStream_t st);

// Tridiagonalise all blocks (A overwritten by the reflectors, lower part). Full symmetric
// storage is required on input.
void launch_tridiag_batched(const BatchDesc &bd, double *A, double *d, double *e, double *tau,
                            int nmax, cudaStream_t st);

// Eigenvalues. mode 0: all n eigenvalues of each block into w (ascending), cnt[b] = n.
// mode 1: eigenvalues below `cut` (strict `<`) ; mode 2: eigenvalues `<= cut`. Counts go to
// cnt[b]; w receives the selected eigenvalues ascending.
void launch_eigvals_batched(const BatchDesc &bd, const double *d, const double *e, double *w,
                            int *cnt, int mode, double cut, cudaStream_t st);

// Eigenvectors of eigenvalues w[voff[b] + 0 .. sel[b]-1]: written to Z + zoff[b] with
// leading dimension zld[b] (column-major, one column per eigenvalue). `work` needs
// 6 * sum_b(n[b]) * 256 doubles at most (see eigvecs_work_doubles).
void launch_eigvecs_batched(const BatchDesc &bd, const double *A, const double *d,
                            const double *e, const double *tau, const double *w,
                            const int *sel, const long long *zoff, const int *zld, double *Z,
                            double *work, const long long *workoff, int nmax, int *err,
                            cudaStream_t st);

// Same output as launch_eigvecs_batched (n <= 1024), without work buffer: inverse iteration
// with the factors in shared memory (one warp per cluster) and a blocked back-transformation.
// Both set *err = 1 (err may be null) when inverse iteration fails its growth test for some
// vector (dstein's convergence criterion); the flag is never cleared by the kernels.
// Diagnostics of the fast batched inverse iteration: the first vector that failed its growth
// test since the last clear ({failed, block, eigenvalue index, block order}).
void invit_fail_clear(cudaStream_t st);
void invit_fail_info(cudaStream_t st, int out[4]);
void launch_eigvecs_batched_fast(const BatchDesc &bd, const double *A, const double *d, const double *e,
                                 const double *tau, const double *w, const int *sel, const long long *zoff,
                                 const int *zld, double *Z, int nmax, int *err, cudaStream_t st);

}  // namespace dvr3d
