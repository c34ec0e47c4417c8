// pes.cuh -- device potential energy surfaces (replacement of the POTV plugin call).
//
// The reference evaluates SUBROUTINE POTV(V,R1,R2,XCOS) once per grid point inside its
// block builders (mkham1 :2178-2183, blc2d1 :3199,:3204). On the device the same values
// are produced inside the block-build kernels: either from the closed-form family below
// or from a table the host filled with its own POTV at the DVR grid.
#pragma once

#include "../../include/dvr3d_b200.h"

namespace dvr3d {

struct PesParams {
    int kind;              // dvr3d_pes_kind
    double p[DVR3D_PES_MORSE_SUM_NPARAM];
    const double *grid;    // DVR3D_PES_GRID: v[(ia*npnt2 + i2)*npnt1 + i1]
    int npnt1, npnt2;
};

// DVR3D_PES_MORSE_SUM; same formula and operation order as the host-side definition.
__host__ __device__ __forceinline__ double pes_morse_sum(const double *p, double r1, double r2, double x) {
    const double d1 = r1 - p[2], d2 = r2 - p[5];
    const double m1 = 1.0 - exp(-p[1] * d1);
    const double m2 = 1.0 - exp(-p[4] * d2);
    const double x2 = x * x;
    const double P1 = x, P2 = 0.5 * (3.0 * x2 - 1.0), P3 = 0.5 * (5.0 * x2 - 3.0) * x;
    const double P4 = (35.0 * x2 * x2 - 30.0 * x2 + 3.0) / 8.0;
    const double dc = x - p[7];
    return p[0] * m1 * m1 + p[3] * m2 * m2 + p[6] * dc * dc + p[8] * d1 * d2 + p[9] * P1 +
           p[10] * P2 + p[11] * P3 + p[12] * P4;
}

// V at grid point (i1 of r1, i2 of r2, ia of the angular grid).
__device__ __forceinline__ double pes_eval(const PesParams &P, double r1, double r2, double x,
                                           int i1, int i2, int ia) {
    if (P.kind == DVR3D_PES_GRID) return P.grid[((size_t)ia * P.npnt2 + i2) * P.npnt1 + i1];
    return pes_morse_sum(P.p, r1, r2, x);
}

}  // namespace dvr3d
