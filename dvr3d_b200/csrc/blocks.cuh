// blocks.cuh -- parameters and launchers of the block-build and basis-transform kernels.
#pragma once

#include <cuda_runtime.h>

#include "pes.cuh"

namespace dvr3d {

// Radau (idia = -2) 2D blocks: one per angle, n = npnt (npnt + 1 - 2 ipar) / 2.
struct RadauBuild {
    int n, npnt, ipar, jrot, kz;
    int zperp;                // z axis perpendicular to the plane: z_blc2d1's J > 0 terms
    const int *pa, *pb;       // pair -> (alpha, beta) radial indices, 0-based
    const double *r;          // radial grid (npnt)
    const double *hr;         // DVR kinetic matrix xk1 (npnt x npnt)
    const double *xalf;       // cos theta of each angle
    double term, term2, term3, urr1;
    double xterm;             // ZX: k^2 (1/ur1 - 1/urr1), subtracted over (1 - x^2) (blc2d1 :3169)
    PesParams pes;
};

// Jacobi 1D blocks: npntc * npntb blocks of dimension npnta.
struct Jacobi1D {
    int npnta, npntb, npntc, ztheta, zr2r1, zembed, jrot;
    const double *r1, *r2, *xalf;
    const double *ta;         // kinetic matrix of coordinate a (xk1, xk2 or L), lda
    int lda;
    double ur1, ur2, urr1, urr2, term;
    double w3k;               // ZX, theta first: k^2 of mkham1's extra term (:2166-2171), else 0
    PesParams pes;
};

// Jacobi 2D blocks: one per point of coordinate c.
struct Jacobi2D {
    int npnta, npntb;
    const int *n2;            // [npntc] 2D dimension (sum of kept 1D states)
    const long long *uoff;    // [npntc] offset of U (npnta x n2) in U
    const double *U;          // selected 1D eigenvectors, columns
    const int *bidx;          // [sum n2] coordinate-b index of each 1D state
    const long long *e1off;   // [npntc] offset into e1 / bidx
    const double *e1;         // [sum n2] 1D eigenvalues
    const double *tb;         // kinetic matrix of coordinate b, ldb
    int ldb;
    const long long *hoff;    // [npntc] offset of H2 block (n2 x n2)
};

struct CTrans {
    const int *s2;            // [npntc] selected 2D count
    const long long *v2off;   // [npntc] offset of V2 block (n2 x s2)
    const int *gstart;        // [npntc * (npntb+1)] start of each b group within 1..n2
    const long long *col0;    // [npntc] first column of the block in Vt
    const double *sw;         // [P] sqrt(w) row scaling (1 for theta-first)
    long long ldv;            // leading dimension of Vt (P rounded up, zero padded)
};

void launch_radau_build(const RadauBuild &rb, int nalf, double *H, cudaStream_t st);
void launch_jacobi_build1d(const Jacobi1D &jb, int nblk, double *H, cudaStream_t st);
void launch_jacobi_build2d(const Jacobi2D &jb, int nblk, int n2max, double *H2, cudaStream_t st);
void launch_jacobi_ctrans(const Jacobi2D &jb, const CTrans &ct, int nblk, int s2max,
                          const double *V2, double *Vt, cudaStream_t st);
void launch_scale_rows(double *Vt, int P, long long ncol, const double *sw, cudaStream_t st);
void launch_gather(const double *src, const long long *map, double *dst, long long n, cudaStream_t st);

}  // namespace dvr3d
