// chol.cuh -- FP64 Cholesky factorisation fused with the triangular inverse, on the device.
#pragma once

#include <cuda_runtime.h>

namespace dvr3d {

constexpr int kCholNb = 64;  // block size of the factorisation and of the inverse

// A (n x n, lda even, 16-byte aligned) <- lower triangle of H - sigma I with zeros above
// the diagonal; H is full symmetric storage with leading dimension ldh.
cudaError_t launch_shift_copy_lower(const double *H, long long ldh, int n, double sigma, double *A, long long lda,
                                    cudaStream_t st);

// In place: the lower triangle of the SPD matrix A (upper triangle zero) is replaced by
// inv(L), A = L L^T (recursive; the upper triangle stays zero). work: chol_work_doubles(n)
// doubles. A pivot that is not positive sets *err = kDevNotPosDef; the remaining kernels of
// the factorisation then return at once and the host reads the flag.
size_t chol_work_doubles(int n);
// Products of the recursion large enough for it (ozaki_profitable) may run as FP64-accurate
// int8-sliced tensor-core GEMMs (ozaki.cu) with nslice slices in the given workspace
// (chol_ozaki_work_bytes(n, nslice) bytes, 1 KB aligned); launches counts them.
struct CholOzaki {
    void *work = nullptr;
    size_t bytes = 0;
    int nslice = 8;
    int launches = 0;
};
size_t chol_ozaki_work_bytes(int n, int nslice);
cudaError_t launch_potrf_inv_lower(double *A, long long lda, int n, double *work, int *err, cudaStream_t st,
                                   CholOzaki *oz = nullptr);

// Cholesky of one small SPD matrix G (b x b <= 64, ld b, lower read), in place, and the
// inverse of its factor into ginv (ld 64). A pivot <= rel_tol * max diag(G) (or not finite)
// sets *err = kDevNotPosDef.
cudaError_t launch_chol_small(double *G, int b, double *ginv, double rel_tol, int *err, cudaStream_t st);

}  // namespace dvr3d
