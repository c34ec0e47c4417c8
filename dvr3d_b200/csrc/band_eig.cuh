// band_eig.cuh -- lowest eigenpairs of a symmetric band matrix by bulge chasing to
// tridiagonal form (the projected matrix of the block Krylov solve is block tridiagonal,
// half-bandwidth = the Krylov block size).
#pragma once

#include <cuda_runtime.h>

namespace dvr3d {

constexpr int kBandMaxBw = 32;  // widest band handled (one warp lane per row of a block)

struct BandTri {
    double *A;              // n x n, lower triangle holds the band; rows up to 2b below the
    long long lda;          // diagonal are used as bulge space (zeroed by launch_band_prepare)
    int n, b;
    int ntmax;              // tasks per sweep at most: (n - 2) / b + 1
    double *d, *e;          // out: tridiagonal (d[i] = A[i][i], e[i] = A[i+1][i])
    double *vs;             // out: reflectors, [n - 2][ntmax][kBandMaxBw] (v[0] = 1 stored)
    double *taus;           // out: [n - 2][ntmax]
    unsigned int *progress; // [n] tasks finished per sweep (zeroed by the launcher)
    int *err;
    long long *prof;        // optional [5]: clock cycles of the chase's thread 0 summed over
                            // CTAs (sweep start, reflector, O_s part with the hand-off,
                            // end-of-task wait, unused), or null
    unsigned long long wait_limit;  // polls of one hand-off wait before it gives up (0: 2^24)
};

// Zeroes the bulge space (lower triangle, b < i - j <= 2b) and records the largest dropped
// entry beyond the band and the largest entry inside it (as double bits, both >= 0).
cudaError_t launch_band_prepare(double *A, long long lda, int n, int b, unsigned long long *maxbits2,
                                cudaStream_t st);
size_t band_reflector_doubles(int n, int b);  // vs
size_t band_tau_doubles(int n, int b);        // taus
// Bulge chasing (one CTA per sweep in flight, sweeps pipelined through progress flags),
// then d and e from the reduced matrix.
cudaError_t launch_band_chase(BandTri &t, cudaStream_t st);
// Z (n x nev, ldz) <- Q Z with Q the product of the chase's reflectors (A = Q T Q^T).
cudaError_t launch_band_backtransform(const BandTri &t, double *Z, long long ldz, int nev, cudaStream_t st);

// Lowest eigenpairs without the reduction (band_bisect.cu): Gershgorin bounds and max |A|
// into bounds[0..2]; Sturm-count bisection for the nev lowest eigenvalues into w (one warp
// each, LDL^T of A - sigma I); inverse iteration per cluster of eigenvalues (clusters given by
// cstart[0..ncl], ascending) into the columns of Z, with scratch of
// band_bisect_scratch_doubles(n, b, ncl) doubles; *err = 1 when a vector's growth stays below
// gmin. A: lower band of a symmetric matrix, column-major, half-bandwidth b <= kBandMaxBw.
size_t band_bisect_scratch_doubles(int n, int b, int nclusters);
cudaError_t launch_band_bounds(const double *A, long long lda, int n, int b, double *bounds, cudaStream_t st);
cudaError_t launch_band_bisect(const double *A, long long lda, int n, int b, int nev, const double *bounds, double *w,
                               cudaStream_t st);
cudaError_t launch_band_invit(const double *A, long long lda, int n, int b, const double *w, const int *cstart, int ncl,
                              const double *bounds, double *scratch, double *Z, long long ldz, double gmin, int *err,
                              cudaStream_t st);

}  // namespace dvr3d
