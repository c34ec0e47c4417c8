// host_setup.h -- host-side set-up of one DVR3DRJZ k block (no GPU work).
//
// Covers the reference's input reading and the small FP64 set-up that precedes the hot
// loops of source/dvr3drjz_segmented.f90: insize (:171-638), setcon (:1016-1188), setfac/
// norms (:1191-1287), lagpt/laguer/lgroot/lgrecr (:1290-1492), keints (:1495-1535), k1k2
// (:1603-1632), jacobi/root/recur/allpts (:1635-1772), asleg (:1775-1843), lmatrx
// (:1846-1911) and the k-loop bookkeeping of ccmain (:810-998). All of it is O(n^3) or
// smaller in n <= 128 and runs once per solve; the hot path lives in the CUDA kernels.
#pragma once

#include <string>
#include <vector>

#include "../../include/dvr3d_b200.h"

namespace dvr3d {

struct HostError {
    int code;
    std::string msg;
};

// Everything the device pipeline needs for one k block.
struct BlockPlan {
    // sizes (COMMON /size/ after insize and the k loop)
    int npnt1 = 0, npnt2 = 0, nalf = 0, idvr = 0, nidvr = 0, maxleg = 0, neval = 0;
    int jrot = 0, kmin = 0, idia = 0, ipar = 0, kz = 0, kd = 0, ku = 0, lincr = 0;
    int max2d = 0, max3d = 0, npnta = 0, npntb = 0, npntc = 0;
    bool radau = false;   // idia == -2: nfmain path
    bool ztheta = false, zr2r1 = true, zcut = false, zall = false, zembed = true, zlin = false;
    bool zrot = false;
    bool zperp = false;   // z axis perpendicular to the plane (mkmain :3934 instead of nfmain)
    int iq = 0;           // z-perp Q symmetry (insize :255-261)
    double alf = 0;       // z-perp Gauss-Jacobi exponent alpha = beta of this k (:945)
    // masses and radial constants (setcon)
    double g1 = 0, g2 = 0, ur1 = 0, ur2 = 0, urr1 = 0, urr2 = 0;
    double beta1 = 0, a1 = 0, beta2 = 0, a2 = 0;
    int iu1 = 0, iu2 = 0;
    double emax1_au = 0, emax2_au = 0;
    // grids
    std::vector<double> r1, r2;        // radial DVR points (bohr)
    std::vector<double> y1, w1, y2, w2; // Gauss-Laguerre points / weights (before sqrt)
    double csx1 = 0, csa1 = 0, tsx1 = 0, tsa1 = 0, csx2 = 0, csa2 = 0, tsx2 = 0, tsa2 = 0;
    std::vector<double> xhalf, whalf;  // Gauss-(associated) Legendre half range
    double cswalf = 0, tswalf = 0;
    std::vector<double> xalf, walf;    // angular grid (idvr points, walf = sqrt(scale w))
    // kinetic matrices, column-major
    std::vector<double> xk1, xk2;      // npnt1^2, npnt2^2
    std::vector<double> xlmatr;        // idvr^2
    // pleg(j, i) * walf(i), j = 0..maxleg, i < nidvr, column-major ((maxleg+1) x nidvr): the
    // angular record of the wavefunction file (:976); orders asleg does not form are zero
    std::vector<double> pleg_walf;
    // J > 0 terms
    double term = 0;                   // jhmain :1970
    double xp0 = 0;                    // the rotational x-term (ZX, :571-577): mkham1 :2166-2171, blc2d1 :3169
    double nf_term = 0, nf_term2 = 0, nf_term3 = 0;  // nfmain :3055-3064; z-perp: z_blc2d1 :4059-4073
                                                     // (k^2/4, s (J(J+1)-k^2)/4, -+J(J+1)/4)
};

// Reads the job deck text (namelist PRT + cards). Throws HostError.
void parse_deck(const std::string &text, dvr3d_deck &d);

// insize + setcon + ccmain set-up for loop index kk. Throws HostError.
void plan_block(const dvr3d_deck &d, int kk, BlockPlan &p);

// k-loop bounds (kd, ku) of ccmain :811-819 for a deck.
void k_range(const dvr3d_deck &d, int &kd, int &ku);

}  // namespace dvr3d
