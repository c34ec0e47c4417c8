// eig_dense.cuh -- FP64 eigensolver for the final Hamiltonian (lowest levels).
#pragma once

#include <cuda_runtime.h>

#include "common.cuh"

namespace dvr3d {

struct DenseTri {
    double *A;          // n x n (lower triangle used), ld = lda (multiple of 8); reflector k
    long long lda;      // is left in A[k+2:, k] (v_{k+1} = 1 implied)
    int n;
    double *d, *e, *tau;          // [n]
    double *V, *W;                // n x nbmax panels (ld = n)
    double *acol, *ybuf;          // [n]
    double *P;                    // symmetric-product partial sums, NT * NT * 64
    double *part;                 // [grid * (2 + 2 nbmax)]
    int NT;                       // number of 64-row blocks covering n
    int j0, nb, nbmax;            // current panel
    GridBarrier *bar;             // zeroed before the first panel
    unsigned int bar_base;        // barrier arrivals made by earlier panels (set by the launcher)
    int *err;
    long long *prof;              // optional [6] phase clock accumulators (CTA 0), or null
    cudaEvent_t *ev;              // optional event pool timing each panel launch (2 per panel)
    int nev;
    int npanel;                   // out: panel launches made
    int cache_tiles;              // > 0: resident mode, tiles kept in shared memory per CTA
    unsigned long long wait_limit;  // polls of one grid-barrier wait before it gives up (0: 2^26)
};

// Resident mode for small matrices: returns the tiles per CTA (0: not applicable) and the
// grid to launch with.
int dense_resident_plan(int device, int n, int *grid);

int dense_tridiag_grid(int device);
int dense_panel_width();
cudaError_t launch_dense_tridiag(DenseTri &t, int grid, cudaStream_t st);
// info[0..3] = lower bound, upper bound, pivmin, ||T||
void launch_dense_eigvals(const double *d, const double *e, int n, int nev, double *e2, double *info,
                          double *w, cudaStream_t st);
// Eigenvectors of the reduced matrix for the nev eigenvalues w, back-transformed into Z.
// Inverse iteration runs with its factors in shared memory when invit_smem_bytes(n) <=
// kInvitSmemMax (else from fac, 5 n T doubles, and X, n nev doubles); the back-transform is
// blocked (GEMM) when bt_work (dense_bt_work_doubles(n, nev)) is given and ldz is even.
constexpr int kInvitSmemMax = 200 * 1024;
size_t invit_smem_bytes(int n);
size_t dense_bt_work_doubles(int n, int nev);
// Eigenvectors of the tridiagonal (d, e) for the nev eigenvalues w into Z (no back-transform);
// eigenvalues closer than ortol_rel ||T|| are orthogonalised as a cluster (1e-6 for the dense
// path; the projected Krylov matrix, whose wanted eigenvalues are graded over orders of
// magnitude, uses a far smaller one so they are not all one cluster).
void launch_tridiag_eigvecs(const double *d, const double *e, int n, const double *w, int nev, const double *info,
                            int *cstart, int *ncl, double *fac, int T, double *X, double *Z, long long ldz,
                            double ortol_rel, cudaStream_t st);
void launch_dense_eigvecs(const double *A, long long lda, int n, const double *d, const double *e,
                          const double *tau, const double *w, int nev,
                          const double *info, int *cstart, int *ncl, double *fac, int T, double *X,
                          double *Z, long long ldz, double *bt_work, cudaStream_t st);
cudaError_t launch_dense_backtransform(const double *A, long long lda, int n, const double *tau, double *Z,
                                       long long ldz, int nev, double *work, cudaStream_t st);

}  // namespace dvr3d
