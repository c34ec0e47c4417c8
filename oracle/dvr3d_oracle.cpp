// dvr3d_oracle.cpp -- CPU FP64 restatement of the DVR3DRJZ hot path (the oracle).
//
// TEST INFRASTRUCTURE ONLY: the checker used by tests/, __graft_entry__.smoke() and the
// CPU-baseline leg of bench.py. The product library never links or calls it.
//
// Every routine below restates the routine of the reference file
// source/dvr3drjz_segmented.f90 named in its comment (line numbers of that file), keeping
// its loop order and arithmetic so its FP64 results agree with the reference to rounding.
// Scratch Fortran units of the reference (ivecs1, ieigs1, ivint, iband, intvec ...) are
// replaced by in-memory arrays holding the same records. LAPACK dsyev is resolved at run
// time from a shared object (scipy's OpenBLAS), as the reference links LAPACK.

#include "dvr3d_oracle.h"

#include <dlfcn.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <thread>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

// ------------------------------------------------------------------ LAPACK binding
typedef void (*dsyev_t)(const char *, const char *, const int *, double *, const int *,
                        double *, double *, const int *, int *, size_t, size_t);
typedef void (*dsyevd_t)(const char *, const char *, const int *, double *, const int *,
                         double *, double *, const int *, int *, const int *, int *, size_t,
                         size_t);
dsyev_t g_dsyev = nullptr;
dsyevd_t g_dsyevd = nullptr;

struct Fail {
    int code;
};
[[noreturn]] void fail(int code) { throw Fail{code}; }

const double autocm = 2.19474624e+05;  // diag3d :2681, cut1d :2895
const double amtoau = 1.8228883e03;    // setcon :1037

// diag(ham,maxham,nham,eig) :2638-2659: dsyev('V','L',nham,ham,maxham,eig,work,3*maxham)
void diag(double *ham, int maxham, int nham, double *eig, int mode = 0) {
    if (nham <= 0) return;
    int info = 0;
    if (mode == 1 && g_dsyevd) {
        int lwork = 1 + 6 * nham + 2 * nham * nham, liwork = 3 + 5 * nham;
        std::vector<double> work(lwork);
        std::vector<int> iwork(liwork);
        g_dsyevd("V", "L", &nham, ham, &maxham, eig, work.data(), &lwork, iwork.data(),
                 &liwork, &info, 1, 1);
    } else {
        if (!g_dsyev) fail(DVR3D_ERR_ARG);
        int lwork = 3 * maxham;
        std::vector<double> work(lwork);
        g_dsyev("V", "L", &nham, ham, &maxham, eig, work.data(), &lwork, &info, 1, 1);
    }
    // the reference only prints ifail (:2656); a failed LAPACK call is reported here
    if (info != 0) fail(DVR3D_ERR_NOCONV);
}

// ------------------------------------------------------------------ problem state
struct Run {
    // COMMON /size/
    int npnt1, npnt2, nalf, nmax1, nmax2, maxleg, nalf2, idvr, npnt, nlim1, nlim2, neval;
    int ncoord, jrot, kmin, idia, ipar, max2d, max3d, max2d2, max3d2, npnta, npntb, npntc;
    int ndima, ndimb, ndimc;
    double emax1, emax2;
    // COMMON /outp/ (hot-path subset)
    bool zrot, zembed, zmors1, zmors2, zcut, zall, zlin, zladd, zquad2, ztheta, zr2r1;
    bool zbisc, zperp, ztwod, zladd_;
    int iq = 0;        // z-perp Q symmetry (insize :255-261)
    double alf = 0.0;  // z-perp Gauss-Jacobi exponent alpha = beta of this k (ccmain :945-947)
    // COMMON /oupb/
    double xp0, xp1, xp2;
    // COMMON /split1/, /split2/, /mass/
    double re1, diss1, we1, beta1, ur1, urr1, a1;
    int iu1;
    double re2, diss2, we2, beta2, ur2, urr2, a2;
    int iu2;
    double xmass[3], xmassr[3], g1, g2;
    // ccmain arrays
    std::vector<double> r1, r2, wt1, wt2, y1, y2, xk1, xk2;  // xk column-major npnt x npnt
    double csx1 = 0, csa1 = 0, tsx1 = 0, tsa1 = 0, csx2 = 0, csa2 = 0, tsx2 = 0, tsa2 = 0;
    // per-k
    int kz, kd, ku, nidvr, nang, nang2, lincr;
    std::vector<double> xalf, walf, xhalf, whalf, xlmatr, pleg;  // xlmatr idvr x idvr
    double cswalf = 0, tswalf = 0;
    // potential
    int pes_kind = 0;
    std::vector<double> pes;
    const double *vgrid = nullptr;
    size_t nvgrid = 0;
    // unit boundary of a stepwise run (oracle_session_*): called before each unit of work of
    // nfmain / jhmain; empty for a plain run
    std::function<void()> gate;
    // selection outcome, published when the selection unit ends (per block: kept 2D states
    // and 2D dimension), for callers of a stepwise run
    std::vector<int> sel_iv2, sel_n2d;
    void tick() const {
        if (gate) gate();
    }
};

// Units of work of one k block for a stepwise run: the gates nfmain / jhmain pass.
int work_units(const Run &R) { return R.idia <= -2 ? 2 * R.nalf + 2 : 4 * R.npntc + 2; }

double pes_morse_sum(const double *p, double r1, double r2, double x) {
    double d1 = r1 - p[2], d2 = r2 - p[5];
    double m1 = 1.0 - std::exp(-p[1] * d1);
    double m2 = 1.0 - std::exp(-p[4] * d2);
    double x2 = x * x;
    double P1 = x, P2 = 0.5 * (3.0 * x2 - 1.0), P3 = 0.5 * (5.0 * x2 - 3.0) * x;
    double P4 = (35.0 * x2 * x2 - 30.0 * x2 + 3.0) / 8.0;
    double dc = x - p[7];
    return p[0] * m1 * m1 + p[3] * m2 * m2 + p[6] * dc * dc + p[8] * d1 * d2 + p[9] * P1 +
           p[10] * P2 + p[11] * P3 + p[12] * P4;
}

// POTV(V,R1,R2,XCOS) plugin (docum.tex:30-47). For a tabulated surface the point is
// identified by its grid indices.
double potv(const Run &R, double r1, double r2, double x, int i1, int i2, int ia) {
    double v;
    if (R.pes_kind == DVR3D_PES_MORSE_SUM) {
        v = pes_morse_sum(R.pes.data(), r1, r2, x);
    } else if (R.pes_kind == DVR3D_PES_GRID) {
        size_t idx = ((size_t)ia * R.npnt2 + i2) * R.npnt1 + i1;
        if (!R.vgrid || idx >= R.nvgrid) fail(DVR3D_ERR_ARG);
        v = R.vgrid[idx];
    } else {
        fail(DVR3D_ERR_ARG);
    }
    if (!std::isfinite(v)) fail(DVR3D_ERR_PES);
    return v;
}

// insize :171-638 (derived sizes only; the printing is omitted) and setcon :1016-1188.
void insize_setcon(Run &R, const dvr3d_deck &d) {
    R.zrot = d.zrot;
    R.zembed = d.zembed;
    R.zmors1 = d.zmors1;
    R.zmors2 = d.zmors2;
    R.zcut = d.zcut;
    R.zall = d.zall;
    R.zlin = d.zlin;
    R.zladd = d.zladd;
    R.zquad2 = d.zquad2;
    R.ztheta = d.ztheta;
    R.zr2r1 = d.zr2r1;
    R.zperp = d.zperp;
    R.ztwod = d.ztwod;
    R.ncoord = d.ncoord;
    R.npnt2 = d.npnt2;
    R.jrot = d.jrot;
    R.neval = d.neval;
    R.nalf = d.nalf;
    R.max2d = d.max2d;
    R.max3d = d.max3d;
    R.idia = d.idia;
    R.kmin = d.kmin;
    R.npnt1 = d.npnt1;
    R.ipar = d.ipar;
    R.max3d2 = d.max3d2;
    R.emax1 = d.emax1;
    R.emax2 = d.emax2;
    for (int i = 0; i < 3; ++i) {
        R.xmass[i] = d.xmass[i];
        R.xmassr[i] = d.xmassr[i];
    }
    if (R.ztwod || d.ncoord == 2) fail(DVR3D_ERR_UNSUPPORTED);
    if (R.zperp && R.idia == 2) fail(DVR3D_ERR_ARG);  // :367-371
    if (!R.zmors1 || !R.zmors2) fail(DVR3D_ERR_UNSUPPORTED);  // keint2 path not restated
    // :241-264
    R.zbisc = false;
    if (R.jrot == 0) {
        R.zembed = true;
        R.kmin = 0;
        R.zrot = false;
    }
    if (R.idia == -2) {
        R.ncoord = 3;
        R.npnt1 = R.npnt2;
        R.idvr = R.nalf;
        R.zmors1 = R.zmors2;
        R.ztheta = false;
        if (R.jrot != 0) R.zbisc = true;
        if (R.zperp) {  // :257-261
            R.iq = R.kmin;
            R.kmin = 1;
            if (R.jrot == 0) R.kmin = 0;
        }
    }
    // the z-perp angular grid has 2 nang2 points in an array of nalf (gaujac at :945); an odd
    // nalf, or a later k block with fewer angles (zladd = F), would read points the reference
    // leaves undefined
    if (R.zperp && (R.idia != -2 || (R.nalf & 1) || !R.zladd)) fail(DVR3D_ERR_UNSUPPORTED);
    R.nalf2 = (R.nalf + 1) / 2;  // :281
    R.ncoord = 3;
    R.maxleg = R.nalf - 1;  // :306-308
    R.nmax2 = R.npnt2 - 1;
    R.nmax1 = R.npnt1 - 1;
    int mi = std::max(1, R.idia);
    if (R.ztheta) {  // :310-328
        R.npnta = R.nalf / mi;
        if (R.zr2r1) {
            R.npntb = R.npnt2;
            R.npntc = R.npnt1;
        } else {
            R.npntb = R.npnt1;
            R.npntc = R.npnt2;
        }
    } else {
        if (R.zr2r1) {
            R.npnta = R.npnt2;
            R.npntb = R.npnt1;
        } else {
            R.npnta = R.npnt1;
            R.npntb = R.npnt2;
        }
        R.npntc = R.nalf / mi;
    }
    if (R.idia == -2) {  // :330-352
        if (R.zrot && (R.jrot + R.kmin) > 1) {
            R.max2d = R.npnt1 * (R.npnt1 + 1) / 2;
            R.max2d2 = R.npnt1 * (R.npnt1 - 1) / 2;
        } else {
            R.max2d = R.npnt1 * (R.npnt1 + 1 - (R.ipar * 2)) / 2;
            R.max2d2 = 0;
        }
        if (!R.zall) R.max3d = std::min(R.max3d, R.max2d * R.nalf);
        if (R.zall) R.max3d = R.max2d * R.nalf;
        if (R.zrot) {
            if (R.max3d2 <= 0) R.max3d2 = R.max3d;
            R.max3d2 = std::min(std::min(R.max3d, R.max2d2 * R.nalf), R.max3d2);
        }
    } else {
        if (R.zall) {
            R.max2d = R.npnta * R.npntb;
            R.max3d = R.max2d * R.npntc;
        } else {
            R.max2d = std::min(R.max2d, R.npnta * R.npntb);
            R.max3d = std::min(R.max3d, R.npnta * R.npntb * R.npntc);
        }
    }
    if (R.neval <= 0) R.neval = 10;  // :354-355
    R.neval = std::min(R.max3d, R.neval);
    if (std::abs(R.idia) == 2) {  // :499-522
        if (R.ipar != 0 && R.ipar != 1) fail(DVR3D_ERR_ARG);
        if (R.idia == 2) {
            R.idvr = R.nalf2;
            if (2 * R.idvr != R.nalf) fail(DVR3D_ERR_ARG);
        }
    } else {
        R.idvr = R.nalf;
        R.ipar = 0;
    }
    if (R.jrot != 0) {  // :523-565
        R.jrot = std::abs(R.jrot);
        if (R.zrot) {
            if (R.kmin != 0 && !R.zbisc) R.kmin = 1;
            if (R.kmin != 0 && R.kmin != 1) R.kmin = 2;
        } else if (std::abs(R.kmin) > std::abs(R.jrot)) {
            fail(DVR3D_ERR_ARG);
        }
        if (R.zbisc) R.zembed = false;
    }
    R.xp0 = d.zx ? 1.0 : 0.0;  // :571-595
    R.xp1 = d.zs0 ? 1.0 : 0.0;
    R.xp2 = d.zs1 ? 1.0 : 0.0;
    R.npnt = std::max(R.npnt1, R.npnt2);  // :602-612
    R.nlim1 = R.npnt1 * (R.npnt1 + 1) / 2;
    R.nlim2 = R.npnt2 * (R.npnt2 + 1) / 2;
    R.ndima = R.npnta;
    if (R.idia <= -2 && !R.zrot) R.ndima = R.ndima - R.ipar;
    R.ndimb = R.npntb;
    R.ndimc = R.npntc;
    if (!R.zquad2) fail(DVR3D_ERR_UNSUPPORTED);  // :618-620 (zquad2=F needs keint2 path)
    if (R.npnt1 < 1 || R.npnt2 < 1 || R.nalf < 1 || R.npnt1 > 120 || R.npnt2 > 120 ||
        R.nalf > 250)
        fail(DVR3D_ERR_ARG);

    // setcon :1070-1160
    if (R.idia >= 1) {
        R.g1 = R.xmass[1] / (R.xmass[1] + R.xmass[2]);
        R.g2 = 0.0;
    } else {
        double a = std::sqrt(R.xmass[2] / (R.xmass[0] + R.xmass[1] + R.xmass[2]));
        double b = R.xmass[1] / (R.xmass[0] + R.xmass[1]);
        R.g1 = 1.0 - a / (a + b - a * b);
        R.g2 = 1.0 - a / (1.0 - b + a * b);
    }
    if (R.xmassr[0] <= 0.0)
        for (int i = 0; i < 3; ++i) R.xmassr[i] = R.xmass[i];  // :1054
    const double *xm = R.xmass, *xr = R.xmassr;
    R.ur1 = amtoau / (R.g2 * R.g2 / xm[0] + 1.0 / xm[1] + (1.0 - R.g2) * (1.0 - R.g2) / xm[2]);
    R.ur2 = amtoau / (1.0 / xm[0] + R.g1 * R.g1 / xm[1] + (1.0 - R.g1) * (1.0 - R.g1) / xm[2]);
    R.urr1 = amtoau / (R.g2 * R.g2 / xr[0] + 1.0 / xr[1] + (1.0 - R.g2) * (1.0 - R.g2) / xr[2]);
    R.urr2 = amtoau / (1.0 / xr[0] + R.g1 * R.g1 / xr[1] + (1.0 - R.g1) * (1.0 - R.g1) / xr[2]);
    R.re1 = d.re1;
    R.diss1 = d.diss1;
    R.we1 = d.we1;
    R.re2 = d.re2;
    R.diss2 = d.diss2;
    R.we2 = d.we2;
    if (R.diss1 <= 0.0 || R.we1 <= 0.0) fail(DVR3D_ERR_ARG);
    R.beta1 = R.we1 * std::sqrt(0.5 * R.ur1 / R.diss1);  // :1123-1125
    R.a1 = 4.0 * R.diss1 / R.we1;
    R.iu1 = (int)(R.a1 + 0.5);
    if (R.idia != -2) {  // :1142-1149
        if (R.diss2 <= 0.0 || R.we2 <= 0.0) fail(DVR3D_ERR_ARG);
        R.beta2 = R.we2 * std::sqrt(0.5 * R.ur2 / R.diss2);
        R.a2 = 4.0 * R.diss2 / R.we2;
        R.iu2 = (int)(R.a2 + 0.5);
    }
}

// norms :1261-1287
void norms(std::vector<double> &dnorm, const std::vector<double> &fact, double &cc,
           double alf, int npnt, int nmax) {
    double count = (double)npnt + alf;
    cc = fact[npnt] / count;  // fact is 1-based in the reference: fact(i) -> fact[i]
    std::vector<double> bin(npnt + 2);
    int npt1 = npnt + 1;
    bin[npt1] = 1.0;
    for (int i = 1; i <= npnt; ++i) {
        int n = npt1 - i;
        bin[n] = bin[n + 1] * count / (double)i;
        count = count - 1.0;
    }
    npt1 = npt1 + 1;
    dnorm.assign(nmax + 1, 0.0);
    for (int i = 0; i <= nmax; ++i) dnorm[i] = std::sqrt(bin[i + 1] * fact[i + 1] * fact[npt1 - i - 1]);
}

// lgrecr :1466-1492 (b, c 1-based)
void lgrecr(double &pn, double &dpn, double &pn1, double x, int nn, double alf,
            const std::vector<double> &b, const std::vector<double> &c) {
    double p1 = 1.0, p = x - alf - 1.0, dp1 = 0.0, dp = 1.0;
    for (int j = 2; j <= nn; ++j) {
        double q = (x - b[j]) * p - c[j] * p1;
        double dq = (x - b[j]) * dp - c[j] * dp1 + p;
        p1 = p;
        p = q;
        dp1 = dp;
        dp = dq;
    }
    pn = p;
    dpn = dp;
    pn1 = p1;
}

// lgroot :1439-1463
void lgroot(double &x, int nn, double alf, double &dpn, double &pn1,
            const std::vector<double> &b, const std::vector<double> &c, double eps) {
    const int itmax = 10;
    int iter = 0;
    for (;;) {
        ++iter;
        double p;
        lgrecr(p, dpn, pn1, x, nn, alf, b, c);
        double d = p / dpn;
        x = x - d;
        if (std::fabs(d / x) <= eps) return;
        if (iter >= itmax) return;  // the reference warns and returns (:1459)
    }
}

static inline double fsign1(double v) { return v >= 0.0 ? 1.0 : -1.0; }

// laguer :1369-1436
void laguer(int nn, std::vector<double> &x, std::vector<double> &a, double alf, double &csx,
            double &csa, double &tsx, double cc) {
    const double eps = 1.0e-12;
    std::vector<double> b(nn + 2), c(nn + 2);
    csx = 0.0;
    csa = 0.0;
    double fa = alf + 1.0;
    b[1] = fa;
    c[1] = 0.0;
    double fn = 1.0;
    for (int j = 2; j <= nn; ++j) {
        fa = fa + 2.0;
        b[j] = fa;
        c[j] = fn * (alf + fn);
        fn = fn + 1.0;
    }
    tsx = fn * (alf + fn);
    double xt1 = 0.0, xt2 = 0.0;
    double xt = (1.0 + alf) * (2.0 + alf) / (1.0 + 3.0 * fn + 2.0 * alf);
    double step = 3.0 * (1.0 + alf) / (1.0 + 3.0 * fn + alf);
    double pt, pt2, dpn, pn1;
    lgrecr(pt, dpn, pn1, xt, nn, alf, b, c);
    x.assign(nn, 0.0);
    a.assign(nn, 0.0);
    for (int i = 1; i <= nn; ++i) {
        if (i <= 2) {
            // smallest two zeros by brute-force search (:1410-1419)
            for (;;) {
                xt2 = xt + step;
                lgrecr(pt2, dpn, pn1, xt2, nn, alf, b, c);
                if (fsign1(pt) * fsign1(pt2) > 0.0) {
                    pt = pt2;
                    xt = xt2;
                    continue;
                }
                pt = pt2;
                xt = 0.5 * (xt + xt2);
                break;
            }
        } else {
            // Stroud & Secrest formula for the other zeros (:1421-1425)
            double fi = (double)(i - 2);
            double rr1 = (1.0 + 2.55 * fi) / (1.9 * fi);
            double rr2 = 1.26 * fi * alf / (1.0 + 3.5 * fi);
            double ratio = (rr1 + rr2) / (1.0 + 0.3 * alf);
            xt = xt + ratio * (xt - xt2);
        }
        lgroot(xt, nn, alf, dpn, pn1, b, c, eps);  // :1427
        xt2 = xt1;
        xt1 = xt;
        x[i - 1] = xt;
        a[i - 1] = cc / dpn / pn1;
        csx = csx + xt;
        csa = csa + a[i - 1];
    }
}

// lagpt :1290-1366 (Morse branch)
void lagpt(std::vector<double> &y, std::vector<double> &r, std::vector<double> &wt,
           std::vector<double> &bass, const std::vector<double> &dnorm, double cc, int npnt,
           int nmax, double re, double beta, double a, int iu, double &csx, double &csa,
           double &tsx, double &tsa) {
    double alf = (double)iu;
    double alfm1 = alf - 1.0;
    laguer(npnt, y, wt, alf, csx, csa, tsx, cc);
    tsa = 1.0 / (dnorm[0] * dnorm[0]);
    r.assign(npnt, 0.0);
    bass.assign((size_t)(nmax + 1) * npnt, 0.0);  // bass(0:nmax, npnt)
    for (int i = 0; i < npnt; ++i) {
        r[i] = re + std::log(a / y[i]) / beta;  // :1322
        double *bs = &bass[(size_t)i * (nmax + 1)];
        bs[0] = 1.0;
        if (nmax >= 1) {
            double amx = alf + 1.0 - y[i];
            bs[1] = amx;
            double en = 1.0;
            for (int n = 2; n <= nmax; ++n) {
                en = en + 1.0;
                amx = amx + 2.0;
                bs[n] = (amx * bs[n - 1] - (alfm1 + en) * bs[n - 2]) / en;
            }
        }
        for (int n2 = 0; n2 <= nmax; ++n2) bs[n2] = bs[n2] * dnorm[n2];
    }
    const double toler = 1.0e-8;  // :1360-1361
    if (std::fabs((csx - tsx) / tsx) > toler) fail(DVR3D_ERR_QUADRATURE);
    if (std::fabs((csa - tsa) / tsa) > toler) fail(DVR3D_ERR_QUADRATURE);
}

// keints :1495-1535 (packed triangle, 0-based)
void keints(std::vector<double> &hbl, double fke, int nmax, int iu) {
    int nlim = (nmax + 1) * (nmax + 2) / 2;
    hbl.assign(nlim, 0.0);
    int index = 0;
    for (int n2 = 1; n2 <= nmax + 1; ++n2) {
        for (int n1 = 1; n1 <= n2; ++n1) {
            if (n1 == n2) {
                hbl[index] = fke * (double)(2 * (n2 - 1) * (n2 + iu) + iu + 1);
            } else if (n1 + 2 == n2) {
                hbl[index] = -fke * std::sqrt((double)((long long)(iu + n1 + 1) * (iu + n1)) *
                                              (double)((n1 + 1) * n1));
            } else {
                hbl[index] = 0.0;
            }
            ++index;
        }
    }
}

// k1k2 :1603-1632 -> xk column-major npnt x npnt
void k1k2(std::vector<double> &xk, const std::vector<double> &hbl,
          const std::vector<double> &bass, const std::vector<double> &wt, int npnt, int nmax) {
    xk.assign((size_t)npnt * npnt, 0.0);
    auto B = [&](int m, int k) { return bass[(size_t)k * (nmax + 1) + m]; };
    for (int k = 0; k < npnt; ++k) {
        for (int kp = 0; kp <= k; ++kp) {
            double wtkkp = wt[k] * wt[kp];
            double acc = 0.0;
            for (int m = 0; m <= nmax; ++m) {
                double t = B(m, k) * wtkkp;
                for (int mp = 0; mp <= nmax; ++mp) {
                    int mx = std::max(m, mp), mn = std::min(m, mp);
                    int in = mx * (mx + 1) / 2 + mn;
                    acc = acc + (hbl[in] * t * B(mp, kp));
                }
            }
            xk[(size_t)kp * npnt + k] = acc;
            xk[(size_t)k * npnt + kp] = acc;
        }
    }
}

// recur :1722-1744 (b, c 1-based)
void recur(double &pn, double &dpn, double &pn1, double x, int nn, double alf, double bta,
           const std::vector<double> &b, const std::vector<double> &c) {
    double p1 = 1.0, p = x + (alf - bta) / (alf + bta + 2.0), dp1 = 0.0, dp = 1.0;
    for (int j = 2; j <= nn; ++j) {
        double q = (x - b[j]) * p - c[j] * p1;
        double dq = (x - b[j]) * dp + p - c[j] * dp1;
        p1 = p;
        p = q;
        dp1 = dp;
        dp = dq;
    }
    pn = p;
    dpn = dp;
    pn1 = p1;
}

// root :1702-1721
void root(double &x, int nn, double alf, double bta, double &dpn, double &pn1,
          const std::vector<double> &b, const std::vector<double> &c, double eps) {
    int iter = 0;
    double p, dp;
    for (;;) {
        ++iter;
        recur(p, dp, pn1, x, nn, alf, bta, b, c);
        double d = p / dp;
        x = x - d;
        if (std::fabs(d) <= eps) break;
        if (iter >= 10) break;
    }
    dpn = dp;
}

// jacobi :1635-1699. The scan step and lower limit are REAL*4 literals in the reference.
void jacobi(int nn, int nn2, std::vector<double> &x, std::vector<double> &a, double alf,
            double bta, double &csa, double tsa) {
    const double eps = 1.0e-12;
    std::vector<double> b(nn + 2), c(nn + 2), xt(nn + 2);
    csa = 0.0;
    c[1] = 0.0;
    b[1] = 0.0;
    for (int i = 2; i <= nn; ++i) {
        double xi = (double)(float)i;
        b[i] = 0.0;
        c[i] = 4.0 * (xi - 1.0) * (alf + xi - 1.0) * (bta + xi - 1.0) * (alf + bta + xi - 1.0) /
               ((alf + bta + 2.0 * xi - 1.0) * (alf + bta + 2.0 * xi - 2.0) *
                (alf + bta + 2.0 * xi - 2.0) * (alf + bta + 2.0 * xi - 3.0));
    }
    double cc = tsa;
    for (int i = 2; i <= nn; ++i) cc = cc * c[i];
    const double step = (double)0.0001f, xstop = (double)(-0.002f);
    int ii = 0;
    double pm1 = 1.0, xxx = 1.0, p, dp, pn1;
    for (;;) {
        recur(p, dp, pn1, xxx, nn, alf, bta, b, c);
        if (pm1 * p < 0.0) {
            pm1 = -pm1;
            ++ii;
            xt[ii] = xxx;
        }
        if (ii == nn2) break;
        xxx = xxx - step;
        if (!(xxx > xstop)) fail(DVR3D_ERR_QUADRATURE);  // :1687-1688
    }
    x.assign(nn2, 0.0);
    a.assign(nn2, 0.0);
    for (int i = 1; i <= nn2; ++i) {
        double dpn;
        root(xt[i], nn, alf, bta, dpn, pn1, b, c, eps);
        x[i - 1] = xt[i];
        a[i - 1] = cc / (dpn * pn1);
        csa = csa + a[i - 1] + a[i - 1];
    }
    if (2 * nn2 != nn) csa = csa - a[nn2 - 1];
}

// allpts :1747-1772
void allpts(Run &R) {
    double scale = (double)std::max(1, R.idia);
    R.xalf.assign(R.idvr, 0.0);
    R.walf.assign(R.idvr, 0.0);
    for (int i = 0; i < R.nang2; ++i) {
        R.xalf[i] = R.xhalf[i];
        R.walf[i] = R.whalf[i];
    }
    for (int i = 1; i <= R.nang2; ++i) {
        R.walf[i - 1] = std::sqrt(scale * R.walf[i - 1]);
        if (R.idia == 2) continue;
        R.xalf[R.nang + 1 - i - 1] = R.xalf[i - 1];
        R.xalf[i - 1] = -R.xalf[i - 1];
        R.walf[R.nang + 1 - i - 1] = R.walf[i - 1];
    }
}

// asleg :1775-1843 -> pleg(0:maxleg, nn2) column-major
void asleg(Run &R) {
    int lmax = R.maxleg, m = R.kz, nn2 = R.nidvr, lincr = R.lincr;
    R.pleg.assign((size_t)(lmax + 1) * nn2, 0.0);
    auto P = [&](int l, int i) -> double & { return R.pleg[(size_t)i * (lmax + 1) + l]; };
    for (int i = 0; i < nn2; ++i) {
        double pmm = 1.0, fact = 1.0;
        for (int j = 1; j <= m; ++j) {
            pmm = -pmm * fact;
            fact = fact + 2.0;
        }
        P(0, i) = pmm;
        double pmmp1 = R.xalf[i] * (m + m + 1) * pmm;
        if (lmax >= 1) P(1, i) = pmmp1;
        int ll = 1;
        for (int l = 2 + m; l <= lmax + lincr; ++l) {
            double r2lm1 = (double)(l + l - 1), rlpmm1 = (double)(l + m - 1), rlmm = (double)(l - m);
            double pll = (R.xalf[i] * r2lm1 * pmmp1 - rlpmm1 * pmm) / rlmm;
            pmm = pmmp1;
            pmmp1 = pll;
            ++ll;
            P(ll, i) = pll;
        }
    }
    std::vector<double> pnorm(lmax + 1);
    int jj = -1;
    for (int j = m; j <= lmax + lincr; ++j) {
        double fact = 1.0;
        for (int i = j - m + 1; i <= j + m; ++i) fact = fact * (double)i;
        double rj = (double)j;
        ++jj;
        pnorm[jj] = std::sqrt((rj + rj + 1.0) / (fact + fact));
    }
    for (int i = 0; i < nn2; ++i) {
        jj = -1;
        for (int j = m; j <= lmax + lincr; ++j) {
            ++jj;
            P(jj, i) = P(jj, i) * pnorm[jj];
        }
    }
}

// the block's angular record of a ZTRAN file (ccmain :972-976) into the trace
void trace_pleg(const Run &R, oracle_trace *tr) {
    if (!tr) return;
    tr->maxleg = R.maxleg;
    tr->nidvr = R.nidvr;
    tr->lincr = R.lincr;
    const size_t n = (size_t)(R.maxleg + 1) * R.nidvr;
    if (!tr->pleg_walf || tr->pleg_cap < n || R.pleg.size() < n) return;
    for (int j = 0; j < R.nidvr; ++j)
        for (int i = 0; i <= R.maxleg; ++i)
            tr->pleg_walf[(size_t)j * (R.maxleg + 1) + i] = R.pleg[(size_t)j * (R.maxleg + 1) + i] * R.walf[j];
}

// lmatrx :1846-1911 -> xlmatr(idvr,idvr) column-major (z-perp: j from 0 with the weights
// (j+1+alf)(j+alf) of the Jacobi polynomials)
void lmatrx(Run &R, int ipar0) {
    int idvr = R.idvr, nidvr = R.nidvr, lmax = R.maxleg;
    R.xlmatr.assign((size_t)idvr * idvr, 0.0);
    int jstart = R.zperp ? 0 : R.kz, iparam = R.zperp ? 0 : R.lincr;
    int jdia = std::max(1, R.idia);
    int jj0 = -jdia;
    if (!R.zperp && jstart % jdia != ipar0) {
        ++jj0;
        ++jstart;
    }
    auto P = [&](int l, int i) { return R.pleg[(size_t)i * (lmax + 1) + l]; };
    for (int k = 0; k < nidvr; ++k) {
        double term = R.walf[k];
        for (int kp = k; kp < nidvr; ++kp) {
            double sumj1 = 0.0;
            int jj = jj0;
            for (int j = jstart; j <= lmax + iparam; j += jdia) {
                jj = jj + jdia;
                if (R.zperp)
                    sumj1 = sumj1 + P(jj, k) * P(jj, kp) * ((j + 1 + R.alf) * (j + R.alf));
                else
                    sumj1 = sumj1 + P(jj, k) * P(jj, kp) * (double)((j + 1) * j);
            }
            double v = sumj1 * term * R.walf[kp];
            R.xlmatr[(size_t)k * idvr + kp] = v;
            R.xlmatr[(size_t)kp * idvr + k] = v;
        }
    }
}

// gammln :4265-4286: log Gamma by the six-term Lanczos series of the reference (the
// coefficients are the reference's; its weights and normalisations carry their ~1e-10 error).
double gammln(double xx) {
    static const double cof[6] = {76.18009173, -86.50532033, 24.01409822, -1.231739516, 0.120858003e-2,
                                  -0.536382e-5};
    const double stp = 2.50662827465;
    double x = xx - 1.0;
    double tmp = x + 5.5;
    tmp = (x + 0.5) * std::log(tmp) - tmp;
    double ser = 1.0;
    for (int j = 0; j < 6; ++j) {
        x = x + 1.0;
        ser = ser + cof[j] / x;
    }
    return tmp + std::log(stp * ser);
}

// gaujac :4190-4263: n Gauss-Jacobi points (descending) and weights for weight
// (1-x)^alf (1+x)^bet; Newton on the three-term recurrence from the reference's initial
// guesses (its 0.012 is a REAL*4 literal).
void gaujac(std::vector<double> &x, std::vector<double> &w, int n, double alf, double bet) {
    const double eps = 3.0e-14;
    const int maxit = 10;
    const double c012 = (double)0.012f;
    double z = 0.0, pp = 0.0, p2 = 0.0, temp = 0.0;
    for (int i = 1; i <= n; ++i) {
        const double dn = (double)n;
        if (i == 1) {
            const double an = alf / dn, bn = bet / dn;
            const double r1 = (1.0 + alf) * (2.78 / (4.0 + (double)(n * n)) + 0.768 * an / dn);
            const double r2 = 1.0 + 1.48 * an + 0.96 * bn + 0.452 * an * an + 0.83 * an * bn;
            z = 1.0 - r1 / r2;
        } else if (i == 2) {
            const double r1 = (4.1 + alf) / ((1.0 + alf) * (1.0 + 0.156 * alf));
            const double r2 = 1.0 + 0.06 * (dn - 8.0) * (1.0 + 0.12 * alf) / dn;
            const double r3 = 1.0 + c012 * bet * (1.0 + 0.25 * std::fabs(alf)) / dn;
            z = z - (1.0 - z) * r1 * r2 * r3;
        } else if (i == 3) {
            const double r1 = (1.67 + 0.28 * alf) / (1.0 + 0.37 * alf);
            const double r2 = 1.0 + 0.22 * (dn - 8.0) / dn;
            const double r3 = 1.0 + 8.0 * bet / ((6.28 + bet) * (double)(n * n));
            z = z - (x[0] - z) * r1 * r2 * r3;
        } else if (i == n - 1) {
            const double r1 = (1.0 + 0.235 * bet) / (0.766 + 0.119 * bet);
            const double r2 = 1.0 / (1.0 + 0.639 * (dn - 4.0) / (1.0 + 0.71 * (dn - 4.0)));
            const double r3 = 1.0 / (1.0 + 20.0 * alf / ((7.5 + alf) * (double)(n * n)));
            z = z + (z - x[n - 4]) * r1 * r2 * r3;
        } else if (i == n) {
            const double r1 = (1.0 + 0.37 * bet) / (1.67 + 0.28 * bet);
            const double r2 = 1.0 / (1.0 + 0.22 * (double)(n - 8) / dn);
            const double r3 = 1.0 / (1.0 + 8.0 * alf / ((6.28 + alf) * (double)(n * n)));
            z = z + (z - x[n - 3]) * r1 * r2 * r3;
        } else {
            z = 3.0 * x[i - 2] - 3.0 * x[i - 3] + x[i - 4];
        }
        const double alfbet = alf + bet;
        for (int its = 1; its <= maxit; ++its) {
            temp = 2.0 + alfbet;
            double p1 = (alf - bet + temp * z) / 2.0;
            p2 = 1.0;
            for (int j = 2; j <= n; ++j) {
                const double p3 = p2;
                p2 = p1;
                temp = 2.0 * (double)j + alfbet;
                const double c1 = 2.0 * (double)j * ((double)j + alfbet) * (temp - 2.0);
                const double c2 = (temp - 1.0) * (alf * alf - bet * bet + temp * (temp - 2.0) * z);
                const double c3 = 2.0 * ((double)(j - 1) + alf) * ((double)(j - 1) + bet) * temp;
                p1 = (c2 * p2 - c3 * p3) / c1;
            }
            pp = (dn * (alf - bet - temp * z) * p1 + 2.0 * (dn + alf) * (dn + bet) * p2) / (temp * (1.0 - z * z));
            const double z1 = z;
            z = z1 - p1 / pp;
            if (std::fabs(z - z1) <= eps) break;
        }
        x[i - 1] = z;
        w[i - 1] = std::exp(gammln(alf + dn) + gammln(bet + dn) - gammln(dn + 1.0) - gammln(dn + alfbet + 1.0)) *
                   temp * std::pow(2.0, alfbet) / (pp * p2);
    }
}

// jac_basis :4136-4154 with jacgt :4158-4186 and norms2 :4288-4308: normalised Jacobi
// polynomials P_i^(alf,bet)(x_n), i = 0..nb, n < nn -> basis (0:nb, nn) column-major
void jac_basis(int nn, int nb, double alf, double bet, const std::vector<double> &x, std::vector<double> &basis) {
    const double lmd = alf + bet + 1.0;
    std::vector<double> norm(nb + 1);
    for (int n = 0; n <= nb; ++n) {
        const double a1 = gammln((double)(n + 1)), a2 = gammln((double)n + lmd);
        const double a3 = gammln((double)n + alf + 1.0), a4 = gammln((double)n + bet + 1.0);
        const double norm1 = std::pow(2.0, -lmd) * (2.0 * (double)n + lmd) * std::exp(a1 + a2 - a3 - a4);
        norm[n] = std::sqrt(norm1);
    }
    std::vector<double> A1(nb + 1), A2(nb + 1), A3(nb + 1), A4(nb + 1);
    for (int n = 1; n <= nb; ++n) {
        A1[n] = 2.0 * (n + 1.0) * (n + lmd) * (2.0 * n + lmd - 1.0);
        A2[n] = (2.0 * n + lmd) * (alf * alf - bet * bet);
        A3[n] = (2.0 * n + lmd - 1.0) * (2.0 * n + lmd) * (2.0 * n + lmd + 1.0);
        A4[n] = 2.0 * (n + alf) * (n + bet) * (2.0 * n + lmd + 1.0);
    }
    basis.assign((size_t)(nb + 1) * nn, 0.0);
    std::vector<double> b(nb + 1);
    for (int i = 0; i < nn; ++i) {
        b[0] = 1.0;
        if (nb >= 1) b[1] = (alf - bet + (lmd + 1.0) * x[i]) / 2.0;
        for (int n = 2; n <= nb; ++n)
            b[n] = ((A2[n - 1] + A3[n - 1] * x[i]) * b[n - 1] - A4[n - 1] * b[n - 2]) / A1[n - 1];
        for (int n = 0; n <= nb; ++n) basis[(size_t)i * (nb + 1) + n] = b[n] * norm[n];
    }
}

// ccmain :641-1013 up to the driver dispatch, for loop index kk.
void ccmain_setup(Run &R, int kk) {
    // setfac :1191-1258
    std::vector<double> fact(R.npnt + 2);
    fact[1] = 1.0;
    double count = 1.0;
    for (int i = 1; i <= R.npnt; ++i) {
        fact[i + 1] = count * fact[i];
        count = count + 1.0;
    }
    std::vector<double> dnorm1, dnorm2, bass1, bass2, hbl1, hbl2;
    double cc1, cc2;
    norms(dnorm1, fact, cc1, (double)R.iu1, R.npnt1, R.nmax1);
    if (R.idia > -2) norms(dnorm2, fact, cc2, (double)R.iu2, R.npnt2, R.nmax2);
    // :764-785
    lagpt(R.y1, R.r1, R.wt1, bass1, dnorm1, cc1, R.npnt1, R.nmax1, R.re1, R.beta1, R.a1, R.iu1,
          R.csx1, R.csa1, R.tsx1, R.tsa1);
    if (R.idia > -2) {
        lagpt(R.y2, R.r2, R.wt2, bass2, dnorm2, cc2, R.npnt2, R.nmax2, R.re2, R.beta2, R.a2,
              R.iu2, R.csx2, R.csa2, R.tsx2, R.tsa2);
        keints(hbl2, R.beta2 * R.beta2 / (8.0 * R.ur2), R.nmax2, R.iu2);
    }
    keints(hbl1, R.beta1 * R.beta1 / (8.0 * R.ur1), R.nmax1, R.iu1);
    std::vector<double> w1 = R.wt1, w2 = R.wt2;  // :797-798 take square roots
    for (auto &w : w1) w = std::sqrt(w);
    for (auto &w : w2) w = std::sqrt(w);
    k1k2(R.xk1, hbl1, bass1, w1, R.npnt1, R.nmax1);  // :802-804
    if (R.idia > -2) k1k2(R.xk2, hbl2, bass2, w2, R.npnt2, R.nmax2);

    // k-loop state of :810-819 and :857-916, replayed up to kk
    if (R.zrot) {
        R.kd = 1 - std::min(R.kmin, 1);
        R.ku = R.jrot;
        if (R.kmin == 2) R.ku = R.ku + 1;
    } else {
        R.kd = R.kmin;
        R.ku = R.kmin;
    }
    if (kk < R.kd || kk > R.ku) fail(DVR3D_ERR_ARG);
    int max2d1 = R.max2d, max3d1 = R.max3d;
    int kkz12 = 0, kkz0 = 0;
    for (int k = R.kd; k <= kk; ++k) {
        if (k <= R.jrot) {
            R.kz = k;
        } else {
            R.kz = 1;
            R.kmin = 0;
            if (!R.zperp) R.ipar = (R.ipar + R.jrot) % 2;
        }
        if (R.zladd || R.kz == R.kd) {
            R.nidvr = R.idvr;
            R.nang = R.nalf;
            R.nang2 = R.nalf2;
            R.lincr = R.kz;
        } else {
            R.lincr = 0;
            if (R.idia != 2) {
                R.nidvr = R.idvr - R.kz;
                R.nang = R.nalf - R.kz;
                R.nang2 = (R.nang + 1) / 2;
            } else if (R.ipar == 0) {
                if (R.kz % 2 == 1) kkz0 += 2;
                R.nidvr = R.idvr - kkz0 / 2;
                R.nang = R.nalf - kkz0;
                R.nang2 = (R.nang + 1) / 2;
            } else {
                if (R.kz % 2 == 0 && R.kz > 0) kkz12 += 2;
                R.nidvr = R.idvr - kkz12 / 2;
                R.nang = R.nalf - kkz12;
                R.nang2 = (R.nang + 1) / 2;
            }
        }
        if (!R.zladd) {
            if (R.ztheta) R.npnta = R.nidvr;
            else R.npntc = R.nidvr;
        }
        if (R.idia <= -2 && R.zrot) {  // :989-998
            if (R.kz > R.kd && !R.zperp) R.ipar = (R.ipar + 1) % 2;
            if (R.ipar > 0) {
                R.max2d = R.max2d2;
                R.max3d = R.max3d2;
            } else {
                R.max2d = max2d1;
                R.max3d = max3d1;
            }
        }
    }
    if (R.zperp) {  // :945-966: Gauss-Jacobi points, Jacobi polynomials, square-rooted weights
        const double rj = (double)R.jrot, rk = (double)R.kz;
        R.alf = std::sqrt(0.5 * ((rj * rj + rj) - rk * rk));
        R.xalf.assign(R.idvr, 0.0);
        R.walf.assign(R.idvr, 0.0);
        gaujac(R.xalf, R.walf, 2 * R.nang2, R.alf, R.alf);
        jac_basis(R.nidvr, R.maxleg, R.alf, R.alf, R.xalf, R.pleg);
        for (int i = 0; i < R.nidvr; ++i) R.walf[i] = std::sqrt(R.walf[i]);
        lmatrx(R, 0);
        return;
    }
    // Gauss-(associated) Legendre points for this k (:887-944)
    double realkz = (double)R.kz;
    R.tswalf = std::pow(2.0, R.kz + R.kz + 1) / (double)(R.kz + 1);
    for (int ia = 1; ia <= R.kz; ++ia) R.tswalf = R.tswalf * (double)ia / (double)(R.kz + ia + 1);
    jacobi(R.nang, R.nang2, R.xhalf, R.whalf, realkz, realkz, R.cswalf, R.tswalf);
    if (std::fabs((R.cswalf - R.tswalf) / R.tswalf) > 1.0e-8) fail(DVR3D_ERR_QUADRATURE);
    allpts(R);
    asleg(R);
    int ipar0 = (R.idia == 2 && R.ipar == 1) ? 1 : 0;
    lmatrx(R, ipar0);
}

// ------------------------------------------------------------------ Radau: nfmain
struct Selected {
    std::vector<double> eigs2d;       // selected 2D eigenvalues (final basis order)
    std::vector<std::vector<double>> vec;  // per block: n2 x count (column-major)
    std::vector<int> count, n2;
};

// blc2d1 :3125-3219 -> ham2 (nham2 x nham2 column-major, full)
void blc2d1(const Run &R, int ig, double xcos, std::vector<double> &ham2, int nham2,
            double term, double term2, double term3, double xtscw) {
    int npnt = R.npnt, ipar = R.ipar;
    const double factr2 = std::sqrt(0.5);
    ham2.assign((size_t)nham2 * nham2, 0.0);
    auto H = [&](int i, int j) -> double & { return ham2[(size_t)(j - 1) * nham2 + (i - 1)]; };
    double xsen2 = 1.0 - xcos * xcos;
    double hfac = 1.0 - R.xp1 * 0.4150706813595e-3 * 1.25;
    auto hrpb = [&](int i, int j) { return R.xk1[(size_t)(j - 1) * R.npnt1 + (i - 1)] * hfac; };
    const std::vector<double> &r = R.r1;
    if (R.jrot != 0) {
        double fact = term + term2 / (1.0 - xcos);
        if (R.kz == 1) fact = fact + term3 * (1.0 + xcos) / (1.0 - xcos);
        int ia = 0;
        double wsum = 0.0, wsum2 = 0.0;
        for (int ibeta = 1; ibeta <= npnt; ++ibeta) {
            for (int ialpha = 1; ialpha <= ibeta - ipar; ++ialpha) {
                double walpha = 0.5 / (r[ialpha - 1] * r[ialpha - 1]);
                double wbeta = 0.5 / (r[ibeta - 1] * r[ibeta - 1]);
                wsum = (walpha + wbeta) * fact / R.urr1 - xtscw;
                wsum2 = R.kz * R.kz * (walpha + wbeta) * (1.0 / R.ur1 - 1.0 / R.urr1) * R.xp0 / xsen2;
                H(ialpha + ia, ialpha + ia) += wsum - wsum2;
            }
            ia = ia + ibeta - ipar;
            if (ipar == 0) H(ia, ia) += wsum - wsum2;
        }
    }
    double q = (ipar == 1) ? -1.0 : 1.0;
    int iap = 0;
    for (int ibetap = 1; ibetap <= npnt; ++ibetap) {
        int ia = 0;
        for (int ibeta = 1; ibeta <= npnt; ++ibeta) {
            for (int ialphp = 1; ialphp <= ibetap - ipar; ++ialphp) {
                for (int ialpha = 1; ialpha <= ibeta - ipar; ++ialpha) {
                    double &h = H(ialphp + iap, ialpha + ia);
                    if (ibeta == ibetap) h = h + hrpb(ialphp, ialpha);
                    if (ibeta == ialphp) h = h + q * hrpb(ibetap, ialpha);
                    if (ialpha == ibetap) h = h + q * hrpb(ialphp, ibeta);
                    if (ialpha == ialphp) h = h + hrpb(ibetap, ibeta);
                    if (ialpha == ialphp && ibeta == ibetap)
                        h = h + potv(R, r[ialpha - 1], r[ibeta - 1], xcos, ialpha - 1, ibeta - 1, ig);
                    if (ialpha == ibetap && ibeta == ialphp)
                        h = h + q * potv(R, r[ibeta - 1], r[ialpha - 1], xcos, ibeta - 1, ialpha - 1, ig);
                    if (ialphp == ibetap) h = h * factr2;
                    if (ialpha == ibeta) h = h * factr2;
                }
            }
            ia = ia + ibeta - ipar;
        }
        iap = iap + ibetap - ipar;
    }
}

// z_blc2d1 :4038-4127 (z-perp embedding, mkmain :3934-4034) -> ham2 (nham2 x nham2)
void z_blc2d1(const Run &R, int ig, double xcos, std::vector<double> &ham2, int nham2) {
    int npnt = R.npnt, ipar = R.ipar;
    const double factr2 = std::sqrt(0.5);
    ham2.assign((size_t)nham2 * nham2, 0.0);
    auto H = [&](int i, int j) -> double & { return ham2[(size_t)(j - 1) * nham2 + (i - 1)]; };
    auto hr = [&](int i, int j) { return R.xk1[(size_t)(j - 1) * R.npnt1 + (i - 1)]; };
    const std::vector<double> &r = R.r1;
    if (R.jrot != 0) {
        const double realj = (double)R.jrot, realkz = (double)R.kz;
        const double term = (R.iq == 0) ? -realj * (realj + 1.0) / 4.0 : realj * (realj + 1.0) / 4.0;
        double fact = (realkz * realkz) / 4.0;
        if (R.kz == 1) fact = fact + term * xcos / (1.0 - xcos * xcos);
        const double s = 1.0 - R.urr1 / R.ur1;
        const double term2 = (realj * realj + realj - realkz * realkz) / 4.0;
        const double fact2 = s * term2 * 1.0 / (1.0 - xcos * xcos);
        int ia = 0;
        double wsum = 0.0, wsum2 = 0.0;
        for (int ibeta = 1; ibeta <= npnt; ++ibeta) {
            for (int ialpha = 1; ialpha <= ibeta - ipar; ++ialpha) {
                const double walpha = 0.5 / (r[ialpha - 1] * r[ialpha - 1] * R.urr1);
                const double wbeta = 0.5 / (r[ibeta - 1] * r[ibeta - 1] * R.urr1);
                wsum = (walpha + wbeta) * fact;
                wsum2 = (walpha + wbeta) * fact2;
                H(ialpha + ia, ialpha + ia) += wsum + wsum2;
            }
            ia = ia + ibeta - ipar;
            if (ipar == 0) H(ia, ia) += wsum + wsum2;
        }
    }
    const double q = (ipar == 1) ? -1.0 : 1.0;
    int iap = 0;
    for (int ibetap = 1; ibetap <= npnt; ++ibetap) {
        int ia = 0;
        for (int ibeta = 1; ibeta <= npnt; ++ibeta) {
            for (int ialphp = 1; ialphp <= ibetap - ipar; ++ialphp) {
                for (int ialpha = 1; ialpha <= ibeta - ipar; ++ialpha) {
                    double &h = H(ialphp + iap, ialpha + ia);
                    if (ibeta == ibetap) h = h + hr(ialphp, ialpha);
                    if (ibeta == ialphp) h = h + q * hr(ibetap, ialpha);
                    if (ialpha == ibetap) h = h + q * hr(ialphp, ibeta);
                    if (ialpha == ialphp) h = h + hr(ibetap, ibeta);
                    if (ialpha == ialphp && ibeta == ibetap)
                        h = h + potv(R, r[ialpha - 1], r[ibeta - 1], xcos, ialpha - 1, ibeta - 1, ig);
                    if (ialpha == ibetap && ibeta == ialphp)
                        h = h + q * potv(R, r[ibeta - 1], r[ialpha - 1], xcos, ibeta - 1, ialpha - 1, ig);
                    if (ialphp == ibetap) h = h * factr2;
                    if (ialpha == ibeta) h = h * factr2;
                }
            }
            ia = ia + ibeta - ipar;
        }
        iap = iap + ibetap - ipar;
    }
}

// nfmain :3006-3121 (mkmain :3934-4034 for the z-perp embedding) with cut2dr :3323-3377, choosr :3223-3319, testiv :3380-3451,
// bloc3d :3455-3505, blc2d2 :3509-3566, vecmul :3570-3595, diag3d :2661-2764.
void nfmain(Run &R, int final_mode, oracle_trace *tr, dvr3d_result *res) {
    auto t0 = std::chrono::steady_clock::now();
    int nalf = R.nalf, npnt = R.npnt, ipar = R.ipar, jrot = R.jrot, kz = R.kz;
    double asw = 0.98205515e-8 * (1.10) * (0.06);
    double bsw = 7.3757478e-9 * (1.10) * (0.06);
    double csw = 1.7082113e-8 * (1.10) * (-0.21);
    double xtscw = ((double)(jrot * jrot + jrot) * (asw + bsw) * 0.5 +
                    (double)(kz * kz) * (csw - (bsw + asw) * 0.5)) * R.xp2;
    double term = 0, term2 = 0, term3 = 0;
    if (jrot != 0) {
        term = (double)(jrot * jrot + jrot - kz * kz) / 8.0;
        term2 = (double)(jrot * jrot + jrot - 3 * kz * kz) / 4.0;
        if (std::abs(kz) == 1) {
            term3 = (double)(jrot * jrot + jrot) / 16.0;
            if (R.kmin >= 1 && R.zrot) term3 = -term3;
        }
    }
    int nham2 = (npnt * (npnt + 1 - ipar * 2)) / 2;
    std::vector<int> nv2(nalf, nham2), iv2a(nalf, 0), iv2b(nalf, 0);  // iv2(1,:), iv2(2,:)
    std::vector<double> ham2, eig2(nham2);
    std::vector<double> eigs2d;
    std::vector<double> vecs2d;  // max2d x (columns), column-major, leading dim nham2
    std::vector<double> eigtmp;
    std::vector<std::vector<double>> allv(nalf), alle(nalf);  // unit intvec (choosr)
    double emaxau = R.emax2 / autocm;
    int npos = 1;
    for (int ig = 0; ig < nalf; ++ig) {
        R.tick();
        if (R.zperp)
            z_blc2d1(R, ig, R.xalf[ig], ham2, nham2);
        else
            blc2d1(R, ig, R.xalf[ig], ham2, nham2, term, term2, term3, xtscw);
        diag(ham2.data(), nham2, nham2, eig2.data());
        if (tr && tr->eig2all && (size_t)(ig + 1) * nham2 <= (size_t)tr->eig2all_cap)
            std::memcpy(tr->eig2all + (size_t)ig * nham2, eig2.data(), sizeof(double) * nham2);
        if (!R.zcut) {
            allv[ig] = ham2;
            alle[ig] = eig2;
            // merge (:3260-3280): equivalent to keeping all eigenvalues sorted
            eigtmp.insert(eigtmp.end(), eig2.begin(), eig2.end());
            std::sort(eigtmp.begin(), eigtmp.end());
        } else {
            int nvec = 0;
            for (int ia = 0; ia < nham2; ++ia) {
                if (eig2[ia] < emaxau) {
                    int ntot = npos + nvec;
                    if (ntot > R.max3d) fail(DVR3D_ERR_CORE_MAX3D);
                    eigs2d.push_back(eig2[ia]);
                    vecs2d.insert(vecs2d.end(), ham2.begin() + (size_t)ia * nham2,
                                  ham2.begin() + (size_t)(ia + 1) * nham2);
                    ++nvec;
                }
            }
            iv2a[ig] = npos;
            iv2b[ig] = nvec;
            npos += nvec;
        }
    }
    R.tick();
    if (!R.zcut) {  // choosr final selection (:3284-3311)
        int itotal = (int)eigtmp.size();
        double emax = (itotal <= R.max3d) ? eigtmp[itotal - 1] : eigtmp[R.max3d - 1];
        int it = 1;
        for (int ig = 0; ig < nalf; ++ig) {
            iv2a[ig] = it;
            int ichose = 0;
            for (int j = 0; j < nv2[ig]; ++j) {
                double e = alle[ig][j];
                if (e <= emax) {
                    eigs2d.push_back(e);
                    vecs2d.insert(vecs2d.end(), allv[ig].begin() + (size_t)j * nham2,
                                  allv[ig].begin() + (size_t)(j + 1) * nham2);
                    ++ichose;
                    ++it;
                }
            }
            iv2b[ig] = ichose;
        }
    }
    // testiv :3380-3451
    if (jrot > 0) {
        int iend = nalf;
        for (int i = nalf / 2; i <= nalf; ++i) {
            if (iv2b[i - 1] == 0) {
                iend = i;
                break;
            }
        }
        for (int i = iend + 1; i <= nalf; ++i) {
            if (iv2b[i - 1] > 0) {
                iv2b[i - 1] = 0;
                iv2a[i - 1] = iv2a[i - 2];
            }
        }
        if (iv2b[nalf - 1] > 0) {
            if (R.zlin) iv2b[nalf - 1] = 0;
            else fail(DVR3D_ERR_THETA0);
        }
    }
    int nham3 = iv2a[nalf - 1] + iv2b[nalf - 1] - 1;  // :3092
    R.sel_iv2 = iv2b;
    R.sel_n2d = nv2;
    auto t1 = std::chrono::steady_clock::now();
    if (final_mode == 3) {
        if (tr) {
            tr->nblocks = nalf;
            tr->nham3 = nham3;
            if (tr->iv2 && tr->iv2_cap >= nalf)
                for (int i = 0; i < nalf; ++i) tr->iv2[i] = iv2b[i];
            tr->stage_s[0] = std::chrono::duration<double>(t1 - t0).count();
        }
        if (res) res->nham3 = nham3;
        return;
    }
    // bloc3d :3455-3505
    std::vector<double> ham3((size_t)nham3 * nham3, 0.0);
    auto V = [&](int col) { return &vecs2d[(size_t)col * nham2]; };
    std::vector<double> hama(nham2);
    int ndim1g = 1;
    for (int ig = 0; ig < nalf; ++ig) {
        R.tick();
        if (iv2b[ig] <= 0) continue;
        int ndim2g = 1;
        for (int igp = 0; igp <= ig; ++igp) {
            if (iv2b[igp] <= 0) continue;
            // blc2d2 :3509-3566 -- nonzero only on the diagonal of the pair basis
            double L = R.xlmatr[(size_t)ig * R.idvr + igp];  // htheta(igammp,igamma)
            const double factr2 = std::sqrt(0.5);
            double q = (ipar == 1) ? -1.0 : 1.0;
            int idx = 0;
            for (int ib = 1; ib <= npnt; ++ib) {
                for (int iaa = 1; iaa <= ib - ipar; ++iaa) {
                    double walpha = 0.5 / (R.r1[iaa - 1] * R.r1[iaa - 1] * R.ur1);
                    double wbeta = 0.5 / (R.r1[ib - 1] * R.r1[ib - 1] * R.ur1);
                    double h = 0.0;
                    double wsum = walpha + wbeta - R.xp1 * 1.5468847900e-8 * 1.250;
                    h = h + L * wsum;
                    if (iaa == ib) h = h + q * L * (walpha + wbeta);
                    if (iaa == ib) h = h * factr2;  // ialphp == ibetap
                    if (iaa == ib) h = h * factr2;  // ialpha == ibeta
                    hama[idx++] = h;
                }
            }
            // vecmul :3570-3595: hamb += va^T hama vb (hama diagonal here)
            int ja0 = ndim1g - 1, jb0 = ndim2g - 1;
            int ca = iv2a[ig] - 1, cb = iv2a[igp] - 1;
            for (int ib = 0; ib < nham2; ++ib) {
                double temp1 = hama[ib];
                if (temp1 == 0.0) continue;
                int ia = ib;
                for (int ja = 0; ja < iv2b[ig]; ++ja) {
                    double temp2 = V(ca + ja)[ia] * temp1;
                    for (int jb = 0; jb < iv2b[igp]; ++jb)
                        ham3[(size_t)(jb0 + jb) * nham3 + (ja0 + ja)] += V(cb + jb)[ib] * temp2;
                }
            }
            ndim2g += iv2b[igp];
        }
        ndim1g += iv2b[ig];
    }
    for (int i = 0; i < nham3; ++i) ham3[(size_t)i * nham3 + i] += eigs2d[i];
    auto t2 = std::chrono::steady_clock::now();
    if (tr) {
        tr->nblocks = nalf;
        tr->nham3 = nham3;
        if (tr->iv2 && tr->iv2_cap >= nalf)
            for (int i = 0; i < nalf; ++i) tr->iv2[i] = iv2b[i];
        if (tr->n2d && tr->n2d_cap >= nalf)
            for (int i = 0; i < nalf; ++i) tr->n2d[i] = nv2[i];
        if (tr->eigs2d && tr->eigs2d_cap >= nham3)
            std::memcpy(tr->eigs2d, eigs2d.data(), sizeof(double) * nham3);
        if (tr->h3 && tr->h3_cap >= (size_t)nham3 * nham3)
            std::memcpy(tr->h3, ham3.data(), sizeof(double) * nham3 * nham3);
    }
    // diag3d :2661-2764
    int meval = std::min(R.neval, nham3);
    std::vector<double> eval(nham3);
    R.tick();
    if (final_mode != 2) diag(ham3.data(), nham3, nham3, eval.data(), final_mode);
    auto t3 = std::chrono::steady_clock::now();
    if (tr) {
        tr->stage_s[0] = std::chrono::duration<double>(t1 - t0).count();
        tr->stage_s[1] = std::chrono::duration<double>(t2 - t1).count();
        tr->stage_s[2] = std::chrono::duration<double>(t3 - t2).count();
        tr->stage_s[3] = std::chrono::duration<double>(t3 - t0).count();
        trace_pleg(R, tr);
    }
    if (tr && tr->psi && final_mode != 2) {
        // transr (:3622-3641): wvfunc(nbass), index over the pairs irs (outer) and the angles
        // with kept states (inner); nbass = iang * max2d
        int iang = 0;
        for (int ig = 0; ig < nalf; ++ig) iang += (iv2b[ig] > 0);
        const long long len = (long long)iang * R.max2d;
        tr->psi_len = len;
        tr->psi_nlev = 0;
        if (tr->psi_cap >= (size_t)len * meval) {
            std::fill(tr->psi, tr->psi + (size_t)len * meval, 0.0);
            for (int l = 0; l < meval; ++l) {
                double *w = tr->psi + (size_t)l * len;
                long long index = 0;
                for (int irs = 0; irs < nham2; ++irs)
                    for (int ig = 0; ig < nalf; ++ig) {
                        if (iv2b[ig] == 0) continue;
                        for (int lev2 = 0; lev2 < iv2b[ig]; ++lev2) {
                            const int ivec2 = iv2a[ig] - 1 + lev2;
                            w[index] += V(ivec2)[irs] * ham3[(size_t)l * nham3 + ivec2];
                        }
                        ++index;
                    }
            }
            tr->psi_nlev = meval;
        }
    }
    if (res) {
        res->nham3 = nham3;
        res->meval = (final_mode == 2) ? 0 : meval;
        res->nblocks = nalf;
        res->kz = R.kz;
        res->ipar = R.ipar;
        if (res->eval && final_mode != 2) {
            if (res->eval_cap < meval) fail(DVR3D_ERR_BUFFER);
            std::memcpy(res->eval, eval.data(), sizeof(double) * meval);
        }
        if (res->iv2 && res->iv2_cap >= nalf)
            for (int i = 0; i < nalf; ++i) res->iv2[i] = iv2b[i];
    }
}

// ------------------------------------------------------------------ Jacobi: jhmain
// mkham1 :2121-2225 -> ham1 (npnta x npnta, column-major, lower filled)
void mkham1(const Run &R, std::vector<double> &ham1, int i1, int i2, double term) {
    int n = R.npnta;
    ham1.assign((size_t)n * n, 0.0);
    auto H = [&](int i, int j) -> double & { return ham1[(size_t)j * n + i]; };
    double wterm = 0.0, w1gama = 0, w2beta = 0, wsum = 0, w3 = 0;
    if (R.ztheta) {
        w1gama = 0.5 / (R.r1[i1] * R.r1[i1] * R.ur1);
        w2beta = 0.5 / (R.r2[i2] * R.r2[i2] * R.ur2);
        wsum = w1gama + w2beta;
        if (R.jrot > 0) {
            if (R.zembed) wterm = term * w2beta * R.ur2 / R.urr2;
            else wterm = term * w1gama * R.ur1 / R.urr1;
            if (R.kz > 0) {
                double s1 = R.ur1 / R.urr1 - 1.0, s2 = R.ur2 / R.urr2 - 1.0;
                w3 = (double)(R.kz * R.kz) * (s1 * w1gama + s2 * w2beta) * R.xp0;
            }
        }
    }
    for (int k = 0; k < n; ++k) {
        double v;
        if (R.ztheta) {
            v = potv(R, R.r1[i1], R.r2[i2], R.xalf[k], i1, i2, k);
        } else if (R.zr2r1) {
            v = potv(R, R.r1[i2], R.r2[k], R.xalf[i1], i2, k, i1);
        } else {
            v = potv(R, R.r1[k], R.r2[i1], R.xalf[i2], k, i1, i2);
        }
        if (R.ztheta) {
            if (R.kz > 0) v = v + w3 / (1.0 - R.xalf[k] * R.xalf[k]);
            H(k, k) = v + wterm;
            for (int kp = 0; kp <= k; ++kp) H(k, kp) = H(k, kp) + R.xlmatr[(size_t)kp * R.idvr + k] * wsum;
        } else {
            if (R.jrot > 0) {
                if (R.zembed) {
                    if (R.zr2r1) wterm = (term * 0.5) / (R.r2[k] * R.r2[k] * R.ur2);
                    else wterm = (term * 0.5) / (R.r2[i1] * R.r2[i1] * R.ur2);
                } else {
                    if (R.zr2r1) wterm = (term * 0.5) / (R.r1[i2] * R.r1[i2] * R.ur1);
                    else wterm = (term * 0.5) / (R.r1[k] * R.r1[k] * R.ur1);
                }
            }
            H(k, k) = v + wterm;
            const std::vector<double> &xk = R.zr2r1 ? R.xk2 : R.xk1;
            int np = R.zr2r1 ? R.npnt2 : R.npnt1;
            for (int kp = 0; kp <= k; ++kp) H(k, kp) = H(k, kp) + xk[(size_t)kp * np + k];
        }
    }
}

// jhmain :1915-2118 with cut1d :2870-2938, mkham2 :2228-2298, cut2d :2941-3003,
// choose :2767-2867, mkham3 :2301-2552, loadh :2554-2609, diag3d :2661-2764.
void jhmain(Run &R, int final_mode, oracle_trace *tr, dvr3d_result *res) {
    auto t0 = std::chrono::steady_clock::now();
    int npnta = R.npnta, npntb = R.npntb, npntc = R.npntc;
    double term = (double)(R.jrot * R.jrot + R.jrot - (2 * R.kz * R.kz));
    // 1D stage (:1973-2003): per ione the selected 1D eigenpairs (units ieigs1/ivecs1)
    std::vector<std::vector<double>> eigs1d(npntc), vecs1d(npntc);  // vecs1d: nham2 x npnta
    std::vector<int> iv1((size_t)npntc * npntb, 0);
    std::vector<double> ham1, eig1(npnta);
    double emax1au = R.emax1 / autocm;
    for (int ione = 0; ione < npntc; ++ione) {
        R.tick();
        std::vector<double> e1;
        std::vector<std::vector<double>> cols;  // each selected vector over npnta
        for (int itwo = 0; itwo < npntb; ++itwo) {
            mkham1(R, ham1, R.zr2r1 ? ione : itwo, R.zr2r1 ? itwo : ione, term);
            diag(ham1.data(), npnta, npnta, eig1.data());
            int ivn = 0;
            if (!R.zall) {
                for (int n = 0; n < npnta; ++n) {
                    if (eig1[n] > emax1au) break;
                    ++ivn;
                }
            } else {
                ivn = npnta;
            }
            iv1[(size_t)ione * npntb + itwo] = ivn;
            for (int i = 0; i < ivn; ++i) {
                if ((int)e1.size() + 1 > R.max2d && !R.zall) fail(DVR3D_ERR_CORE_MAX2D);
                e1.push_back(eig1[i]);
                cols.emplace_back(ham1.begin() + (size_t)i * npnta,
                                  ham1.begin() + (size_t)(i + 1) * npnta);
            }
        }
        int nh = (int)e1.size();
        eigs1d[ione] = e1;
        vecs1d[ione].assign((size_t)nh * npnta, 0.0);  // vecs1d(nham2, ka) column-major
        for (int j = 0; j < nh; ++j)
            for (int ka = 0; ka < npnta; ++ka) vecs1d[ione][(size_t)ka * nh + j] = cols[j][ka];
    }
    // 2D stage (:2019-2053)
    bool zcut = R.zcut || R.zall;
    std::vector<int> ndim2d(npntc, 0), iv2(npntc, 0);
    std::vector<std::vector<double>> eig2s(npntc), vec2s(npntc);  // per block: all or selected
    int low3d = 0;
    double emax2au = R.emax2 / autocm;
    size_t eoff = 0;
    for (int ione = 0; ione < npntc; ++ione) {
        R.tick();
        int nham2 = 0;
        for (int itwo = 0; itwo < npntb; ++itwo) nham2 += iv1[(size_t)ione * npntb + itwo];
        ndim2d[ione] = nham2;
        if (nham2 == 0) continue;
        // mkham2 :2228-2298
        std::vector<double> ham2((size_t)nham2 * nham2, 0.0);
        const std::vector<double> &V1 = vecs1d[ione];
        for (int i3 = 0; i3 < npnta; ++i3)
            for (int j = 0; j < nham2; ++j)
                for (int k = 0; k <= j; ++k)
                    ham2[(size_t)k * nham2 + j] += V1[(size_t)i3 * nham2 + j] * V1[(size_t)i3 * nham2 + k];
        const std::vector<double> *xkb;
        int npb;
        if (R.ztheta) {
            xkb = R.zr2r1 ? &R.xk2 : &R.xk1;
            npb = R.zr2r1 ? R.npnt2 : R.npnt1;
        } else {
            xkb = R.zr2r1 ? &R.xk1 : &R.xk2;
            npb = R.zr2r1 ? R.npnt1 : R.npnt2;
        }
        int ivbsm = 0;
        for (int itwo = 0; itwo < npntb; ++itwo) {
            int ivbpsm = 0, ivb = iv1[(size_t)ione * npntb + itwo];
            for (int itwop = 0; itwop <= itwo; ++itwop) {
                double xkterm = (*xkb)[(size_t)itwop * npb + itwo];
                int ivbp = iv1[(size_t)ione * npntb + itwop];
                for (int j = 0; j < ivb; ++j)
                    for (int jp = 0; jp < ivbp; ++jp)
                        ham2[(size_t)(ivbpsm + jp) * nham2 + (ivbsm + j)] *= xkterm;
                ivbpsm += ivbp;
            }
            ivbsm += ivb;
        }
        for (int nn = 0; nn < nham2; ++nn) ham2[(size_t)nn * nham2 + nn] += eigs1d[ione][nn];
        std::vector<double> eig2(nham2);
        diag(ham2.data(), nham2, nham2, eig2.data());
        if (tr && tr->eig2all && eoff + nham2 <= (size_t)tr->eig2all_cap)
            std::memcpy(tr->eig2all + eoff, eig2.data(), sizeof(double) * nham2);
        eoff += nham2;
        if (zcut) {  // cut2d :2941-3003
            int ivm = 0;
            if (!R.zall) {
                for (int n = 0; n < nham2; ++n) {
                    if (eig2[n] > emax2au) break;
                    ++ivm;
                }
            } else {
                ivm = nham2;
            }
            low3d += ivm;
            if (low3d > R.max3d && !R.zall) fail(DVR3D_ERR_CORE_MAX3D);
            iv2[ione] = ivm;
            eig2s[ione].assign(eig2.begin(), eig2.begin() + ivm);
            vec2s[ione].assign(ham2.begin(), ham2.begin() + (size_t)ivm * nham2);
        } else {
            eig2s[ione] = eig2;
            vec2s[ione] = ham2;
            low3d = R.max3d;
        }
    }
    R.tick();
    if (!zcut) {  // choose :2767-2867
        int nhamsm = 0;
        std::vector<int> ptr(npntc, 1);
        for (int i = 0; i < npntc; ++i) nhamsm += ndim2d[i];
        if (nhamsm < R.max3d) low3d = nhamsm;
        int ipt = 0;
        for (int n = 0; n < low3d; ++n) {
            while (ptr[ipt] > ndim2d[ipt]) ++ipt;
            double eigvib = eig2s[ipt][ptr[ipt] - 1];
            int jpt = ipt;
            for (int j = ipt + 1; j < npntc; ++j) {
                if (ptr[j] > ndim2d[j]) continue;
                if (eig2s[j][ptr[j] - 1] >= eigvib) continue;
                eigvib = eig2s[j][ptr[j] - 1];
                jpt = j;
            }
            ptr[jpt] += 1;
        }
        for (int i = 0; i < npntc; ++i) {
            iv2[i] = ptr[i] - 1;
            eig2s[i].resize(iv2[i]);
            vec2s[i].resize((size_t)iv2[i] * ndim2d[i]);
        }
    }
    int nham3 = low3d;
    R.sel_iv2 = iv2;
    R.sel_n2d = ndim2d;
    auto t1 = std::chrono::steady_clock::now();
    if (final_mode == 3) {
        if (tr) {
            tr->nblocks = npntc;
            tr->nham3 = nham3;
            if (tr->iv1 && tr->iv1_cap >= npntc * npntb)
                std::memcpy(tr->iv1, iv1.data(), sizeof(int) * npntc * npntb);
            if (tr->iv2 && tr->iv2_cap >= npntc)
                for (int i = 0; i < npntc; ++i) tr->iv2[i] = iv2[i];
            if (tr->n2d && tr->n2d_cap >= npntc)
                for (int i = 0; i < npntc; ++i) tr->n2d[i] = ndim2d[i];
            tr->stage_s[0] = std::chrono::duration<double>(t1 - t0).count();
        }
        if (res) res->nham3 = nham3;
        return;
    }
    // mkham3 :2301-2552, first part: cint per block (P x iv2), P = npnta*npntb
    int ncint = npnta * npntb;
    std::vector<std::vector<double>> cint(npntc);
    const bool want_psi = tr && tr->psi;
    std::vector<std::vector<double>> phi(want_psi ? npntc : 0);  // trans: phi before the sqrt(w) scaling
    for (int ione = 0; ione < npntc; ++ione) {
        R.tick();
        int nham2 = ndim2d[ione];
        if (nham2 == 0 || iv2[ione] == 0) continue;
        std::vector<double> &C = cint[ione];
        C.assign((size_t)ncint * iv2[ione], 0.0);
        const std::vector<double> &V1 = vecs1d[ione];
        for (int j = 0; j < iv2[ione]; ++j) {
            const double *h2 = &vec2s[ione][(size_t)j * nham2];
            int ind2 = 0;
            for (int k = 0; k < npnta; ++k) {
                int ind1 = 0;
                for (int itwo = 0; itwo < npntb; ++itwo) {
                    for (int i = 0; i < iv1[(size_t)ione * npntb + itwo]; ++i) {
                        C[(size_t)j * ncint + ind2] += h2[ind1] * V1[(size_t)k * nham2 + ind1];
                        ++ind1;
                    }
                    ++ind2;
                }
            }
            if (want_psi) {
                if (phi[ione].empty()) phi[ione].assign((size_t)ncint * iv2[ione], 0.0);
                std::memcpy(&phi[ione][(size_t)j * ncint], &C[(size_t)j * ncint], sizeof(double) * ncint);
            }
            if (!R.ztheta) {
                int in2 = 0;
                for (int ia = 0; ia < npnta; ++ia) {
                    for (int ib = 0; ib < npntb; ++ib) {
                        int ii1 = R.zr2r1 ? ib : ia, ii2 = R.zr2r1 ? ia : ib;
                        double w1 = 0.5 / (R.r1[ii1] * R.r1[ii1] * R.ur1);
                        double w2 = 0.5 / (R.r2[ii2] * R.r2[ii2] * R.ur2);
                        double wsum = w1 + w2;
                        C[(size_t)j * ncint + in2] *= std::sqrt(wsum);
                        ++in2;
                    }
                }
            }
        }
    }
    // second part: hband = T(ione,ionep) C_ione^T C_ionep; loadh puts it in ham3 (lower)
    std::vector<double> ham3((size_t)nham3 * nham3, 0.0);
    int ivsm = 0;
    for (int ione = 0; ione < npntc; ++ione) {
        R.tick();
        int iv = iv2[ione];
        if (ndim2d[ione] == 0) continue;
        int ivpsm = 0;
        for (int ionep = 0; ionep <= ione; ++ionep) {
            double xkterm;
            if (R.ztheta) {
                xkterm = R.zr2r1 ? R.xk1[(size_t)ionep * R.npnt1 + ione]
                                 : R.xk2[(size_t)ionep * R.npnt2 + ione];
            } else {
                xkterm = R.xlmatr[(size_t)ionep * R.idvr + ione];
            }
            int ivp = iv2[ionep];
            for (int j = 0; j < iv; ++j) {
                const double *cj = &cint[ione][(size_t)j * ncint];
                for (int jp = 0; jp < ivp; ++jp) {
                    const double *cp = &cint[ionep][(size_t)jp * ncint];
                    double h = 0.0;
                    for (int k = 0; k < ncint; ++k) h = h + cj[k] * cp[k] * xkterm;
                    ham3[(size_t)(ivpsm + jp) * nham3 + (ivsm + j)] = h;
                }
            }
            ivpsm += ivp;
        }
        ivsm += iv;
    }
    std::vector<double> eigs2d;
    for (int ione = 0; ione < npntc; ++ione)
        for (int i = 0; i < iv2[ione]; ++i) eigs2d.push_back(eig2s[ione][i]);
    for (int nn = 0; nn < nham3; ++nn) ham3[(size_t)nn * nham3 + nn] += eigs2d[nn];
    auto t2 = std::chrono::steady_clock::now();
    if (tr) {
        tr->nblocks = npntc;
        tr->nham3 = nham3;
        if (tr->iv1 && tr->iv1_cap >= npntc * npntb)
            std::memcpy(tr->iv1, iv1.data(), sizeof(int) * npntc * npntb);
        if (tr->iv2 && tr->iv2_cap >= npntc)
            for (int i = 0; i < npntc; ++i) tr->iv2[i] = iv2[i];
        if (tr->n2d && tr->n2d_cap >= npntc)
            for (int i = 0; i < npntc; ++i) tr->n2d[i] = ndim2d[i];
        if (tr->eigs2d && tr->eigs2d_cap >= nham3)
            std::memcpy(tr->eigs2d, eigs2d.data(), sizeof(double) * nham3);
        if (tr->h3 && tr->h3_cap >= (size_t)nham3 * nham3)
            std::memcpy(tr->h3, ham3.data(), sizeof(double) * nham3 * nham3);
    }
    int meval = std::min(R.neval, nham3);
    std::vector<double> eval(nham3);
    R.tick();
    if (final_mode != 2) diag(ham3.data(), nham3, nham3, eval.data(), final_mode);
    auto t3 = std::chrono::steady_clock::now();
    if (tr) {
        tr->stage_s[0] = std::chrono::duration<double>(t1 - t0).count();
        tr->stage_s[1] = std::chrono::duration<double>(t2 - t1).count();
        tr->stage_s[2] = std::chrono::duration<double>(t3 - t2).count();
        tr->stage_s[3] = std::chrono::duration<double>(t3 - t0).count();
        trace_pleg(R, tr);
    }
    if (want_psi && final_mode != 2) {
        // trans (:3733-3841): psi(idvr, npnt1, npnt2) for each level, summed block by block
        const long long I = R.idvr, n1 = R.npnt1, len = I * R.npnt1 * R.npnt2;
        tr->psi_len = len;
        tr->psi_nlev = 0;
        if (tr->psi_cap >= (size_t)len * meval) {
            std::fill(tr->psi, tr->psi + (size_t)len * meval, 0.0);
            for (int l = 0; l < meval; ++l) {
                double *psi = tr->psi + (size_t)l * len;
                const double *z = &ham3[(size_t)l * nham3];
                int ind2 = 0;
                for (int ic = 0; ic < npntc; ++ic) {
                    for (int j = 0; j < iv2[ic]; ++j, ++ind2) {
                        const double *ph = &phi[ic][(size_t)j * ncint];
                        for (int ia = 0; ia < npnta; ++ia)
                            for (int ib = 0; ib < npntb; ++ib) {
                                long long f;
                                if (!R.ztheta) f = R.zr2r1 ? ic + I * (ib + n1 * ia) : ic + I * (ia + n1 * ib);
                                else f = R.zr2r1 ? ia + I * (ic + n1 * ib) : ia + I * (ib + n1 * ic);
                                psi[f] += z[ind2] * ph[(size_t)ia * npntb + ib];
                            }
                    }
                }
            }
            tr->psi_nlev = meval;
        }
    }
    if (res) {
        res->nham3 = nham3;
        res->meval = (final_mode == 2) ? 0 : meval;
        res->nblocks = npntc;
        res->kz = R.kz;
        res->ipar = R.ipar;
        if (res->eval && final_mode != 2) {
            if (res->eval_cap < meval) fail(DVR3D_ERR_BUFFER);
            std::memcpy(res->eval, eval.data(), sizeof(double) * meval);
        }
        if (res->iv2 && res->iv2_cap >= npntc)
            for (int i = 0; i < npntc; ++i) res->iv2[i] = iv2[i];
    }
}


// ================================================================== ROTLEV3B (second step)
// Restatement of source/rotlev3b_segmented.f90 for one parity (kmin 0 or 1) with the
// Hamiltonian diagonalised in core (dgrot's dsyev path): insize :116-304 (the card),
// select :306-510, radint / mkrad :665-717, angin1 :719-814, angin2 :816-873, jacobi / root /
// recur :941-1049, asleg :1051-1157 (m < 90), solrt :1339-1620, solofd :1682-1729 (its two
// dgemms as loops), loadh :1196-1337 (in-core branch), dgrot :1731-1800.

struct RotFile {
    std::vector<unsigned char> b;
    size_t pos = 0;
    bool eof() const { return pos >= b.size(); }
    // next record's bytes
    std::pair<const unsigned char *, int> rec() {
        if (pos + 4 > b.size()) fail(DVR3D_ERR_ARG);
        int32_t n;
        std::memcpy(&n, &b[pos], 4);
        if (n < 0 || pos + 8 + (size_t)n > b.size()) fail(DVR3D_ERR_ARG);
        std::pair<const unsigned char *, int> r{&b[pos + 4], n};
        pos += 8 + (size_t)n;
        return r;
    }
    void skip() { rec(); }
    std::vector<int> ints() {
        auto r = rec();
        std::vector<int> v(r.second / 4);
        std::memcpy(v.data(), r.first, v.size() * 4);
        return v;
    }
    // getrow: the first n doubles of the next record
    void getrow(double *row, int n) {
        auto r = rec();
        if (r.second < 8 * n) fail(DVR3D_ERR_ARG);
        std::memcpy(row, r.first, 8 * (size_t)n);
    }
};

struct RotBlock {
    int k1, maxleg, nang, lincr, iang, ibass, meval;
    std::vector<double> pleg;  // pleg(ndvr, ndvr) filled with nang*ndvr values (getrow)
    std::vector<int> iv;
    std::vector<double> evib;
    std::vector<double> coef;  // coef(ibass, mvib)
};

// recur :1029-1049
void rot_recur(double &pn, double &dpn, double &pn1, double x, int nn, double alf, double bta,
               const std::vector<double> &b, const std::vector<double> &c) {
    double p1 = 1.0, p = x + (alf - bta) / (alf + bta + 2.0), dp1 = 0.0, dp = 1.0;
    for (int j = 2; j <= nn; ++j) {
        double q = (x - b[j]) * p - c[j] * p1;
        double dq = (x - b[j]) * dp + p - c[j] * dp1;
        p1 = p;
        p = q;
        dp1 = dp;
        dp = dq;
    }
    pn = p;
    dpn = dp;
    pn1 = p1;
}

// jacobi :941-1007 (brute-force sign scan, step 1e-6) with root :1009-1027
void rot_jacobi(int nn, int nn2, std::vector<double> &x, std::vector<double> &a, double alf, double bta,
                double &csa, double tsa) {
    const double eps = 1.0e-12, xstep = 1.0e-6;
    std::vector<double> b(nn + 1, 0.0), c(nn + 1, 0.0), xt(nn + 1, 0.0);
    x.assign(nn + 1, 0.0);
    a.assign(nn + 1, 0.0);
    csa = 0.0;
    for (int i = 2; i <= nn; ++i) {
        double xi = (double)(float)i;
        b[i] = 0.0;
        c[i] = 4.0 * (xi - 1.0) * (alf + xi - 1.0) * (bta + xi - 1.0) * (alf + bta + xi - 1.0) /
               ((alf + bta + 2.0 * xi - 1.0) * (alf + bta + 2.0 * xi - 2.0) * (alf + bta + 2.0 * xi - 2.0) *
                (alf + bta + 2.0 * xi - 3.0));
    }
    double cc = tsa;
    for (int i = 2; i <= nn; ++i) cc = cc * c[i];
    int ii = 0;
    double pm1 = 1.0, xxx = 1.0;
    for (;;) {
        double p, dp, pn1;
        rot_recur(p, dp, pn1, xxx, nn, alf, bta, b, c);
        if (pm1 * p < 0.0) {
            pm1 = -pm1;
            ii = ii + 1;
            xt[ii] = xxx - 0.5 * xstep;
        }
        if (ii == nn2) break;
        xxx = xxx - xstep;
        if (!(xxx > -1.5 * xstep)) fail(DVR3D_ERR_QUADRATURE);
    }
    for (int i = 1; i <= nn2; ++i) {
        double xr = xt[i], p = 0, dp = 0, pn1 = 0, dpn = 0;
        int iter = 0;
        for (;;) {
            iter = iter + 1;
            rot_recur(p, dp, pn1, xr, nn, alf, bta, b, c);
            double d = p / dp;
            xr = xr - d;
            if (std::fabs(d) <= eps) break;
            if (iter >= 10) break;
        }
        dpn = dp;
        x[i] = xr;
        a[i] = cc / (dpn * pn1);
        csa = csa + a[i] + a[i];
    }
    if (2 * nn2 != nn) csa = csa - a[nn2];
}

// asleg :1051-1157 (m < 90): pleg(0:lmax, nn2) column-major
void rot_asleg(std::vector<double> &pleg, int lmax, const std::vector<double> &x, int nn2, int m) {
    if (m < 0 || m >= 90) fail(DVR3D_ERR_UNSUPPORTED);
    pleg.assign((size_t)(lmax + 1) * nn2, 0.0);
    auto P = [&](int l, int i) -> double & { return pleg[(size_t)(i - 1) * (lmax + 1) + l]; };
    for (int i = 1; i <= nn2; ++i) {
        double pmm = 1.0, fact = 1.0;
        for (int j = 1; j <= m; ++j) {
            pmm = -pmm * fact;
            fact = fact + 2.0;
        }
        P(0, i) = pmm;
        double pmmp1 = x[i] * (m + m + 1) * pmm;
        if (lmax >= 1) P(1, i) = pmmp1;
        int ll = 1;
        for (int l = 2 + m; l <= lmax + m; ++l) {
            double r2lm1 = (double)(l + l - 1), rlpmm1 = (double)(l + m - 1), rlmm = (double)(l - m);
            double pll = (x[i] * r2lm1 * pmmp1 - rlpmm1 * pmm) / rlmm;
            pmm = pmmp1;
            pmmp1 = pll;
            ll = ll + 1;
            P(ll, i) = pll;
        }
    }
    std::vector<double> pnorm(lmax + 1);
    int jj = -1;
    for (int j = m; j <= lmax + m; ++j) {
        double fact = 1.0;
        for (int i = j - m + 1; i <= j + m; ++i) fact = fact * std::sqrt((double)i);
        double rj = (double)j;
        jj = jj + 1;
        pnorm[jj] = std::sqrt((rj + rj + 1.0) / 2) / fact;
    }
    for (int i = 1; i <= nn2; ++i)
        for (int j2 = 0; j2 <= lmax; ++j2) P(j2, i) = P(j2, i) * pnorm[j2];
}

struct RotQuad {
    std::vector<double> xalf, walf;  // 1-based, npnt
};

// angin1 :719-814 / angin2 :816-873 -> angmat(iang, iang) column-major (ld iang)
void rot_angin(int step, std::vector<double> &angmat, int iang, const RotQuad &q, int npnt, int ndvr,
               const RotBlock &b1, const RotBlock &b2, int k1, double angfac) {
    const int nang1 = b1.nang, nang2 = b2.nang;
    std::vector<double> plega, plegb;
    rot_asleg(plega, nang1 - 1, q.xalf, npnt, k1);
    rot_asleg(plegb, nang2 - 1, q.xalf, npnt, k1 + step);
    auto PA = [&](int j, int i) { return plega[(size_t)(i - 1) * nang1 + (j - 1)]; };
    auto PB = [&](int k, int i) { return plegb[(size_t)(i - 1) * nang2 + (k - 1)]; };
    std::vector<double> fbr((size_t)ndvr * ndvr, 0.0);
    auto F = [&](int j, int k) -> double & { return fbr[(size_t)(k - 1) * ndvr + (j - 1)]; };
    for (int i = 1; i <= npnt; ++i) {
        double term = step == 1 ? q.walf[i] * (1.0 + q.xalf[i]) : q.walf[i] * ((1.0 + q.xalf[i]) * (1.0 + q.xalf[i]));
        for (int j = 1; j <= nang1; ++j) {
            double fact = term * PA(j, i);
            for (int k = 1; k <= nang2; ++k) F(j, k) = F(j, k) + fact * PB(k, i);
        }
    }
    auto P1 = [&](int j, int i) { return b1.pleg[(size_t)(i - 1) * ndvr + (j - 1)]; };
    auto P2 = [&](int j, int i) { return b2.pleg[(size_t)(i - 1) * ndvr + (j - 1)]; };
    angmat.assign((size_t)iang * iang, 0.0);
    int kkp1 = k1 * (k1 + 1);
    double xkph = (double)k1 + 0.5;
    int i1 = 0;
    for (int i = 1; i <= nang1; ++i) {
        if (b1.iv[i - 1] == 0) continue;
        i1 = i1 + 1;
        int i2 = 0;
        for (int ip = 1; ip <= nang2; ++ip) {
            if (b2.iv[ip - 1] == 0) continue;
            i2 = i2 + 1;
            double sum1 = 0.0, sum2 = 0.0;
            int jj = k1;
            for (int j = 1; j <= nang1; ++j) {
                if (step == 1 && j > 1) {
                    jj = jj + 1;
                    sum1 = sum1 + P1(j, i) * P2(j - 1, ip) * std::sqrt((double)(jj * (jj + 1) - kkp1));
                }
                for (int jp = 1; jp <= nang2; ++jp) sum2 = sum2 + P1(j, i) * P2(jp, ip) * F(j, jp);
            }
            angmat[(size_t)(i2 - 1) * iang + (i1 - 1)] = (step == 1 ? (sum1 + xkph * sum2) : sum2) * angfac;
        }
    }
}

// mkrad :698-717
std::vector<double> rot_mkrad(int nmax, const std::vector<double> &rm2, int iq, int ip, int is) {
    std::vector<double> radmat;
    double symm = (double)(1 - 2 * ip), sign = (double)(1 - 2 * is);
    for (int i1 = 1; i1 <= nmax; ++i1)
        for (int i2 = 1; i2 <= i1 - iq; ++i2) radmat.push_back(sign * (rm2[i2 - 1] + symm * rm2[i1 - 1]));
    return radmat;
}

// solofd :1682-1729 (the two dgemms as loops) -> offdg(mvib2, mvib1)
void rot_solofd(std::vector<double> &offdg, const std::vector<double> &radmat, const std::vector<double> &angmat,
                int iang11, int nmax1, int iq, int iq1, int iq2, int iang1, int iang2, int mvib1, int mvib2,
                const RotBlock &b1, const RotBlock &b2) {
    offdg.assign((size_t)mvib2 * mvib1, 0.0);
    std::vector<double> pdg((size_t)iang1 * mvib2);
    int ir1 = 0, ir2 = 0, ir = 0;
    for (int i1 = 1; i1 <= nmax1; ++i1) {
        for (int i2 = 1; i2 <= i1 - iq; ++i2) {
            int i0 = ir1 * iang1;
            ir1 = ir1 + 1;
            int j0 = ir2 * iang2;
            ir2 = ir2 + 1;
            double rad = radmat[ir];
            ir = ir + 1;
            // pdg = radmat(ir) * angmat * coef2(j0 ...)
            for (int v = 0; v < mvib2; ++v)
                for (int a = 0; a < iang1; ++a) {
                    double s = 0.0;
                    for (int c = 0; c < iang2; ++c)
                        s += angmat[(size_t)c * iang11 + a] * b2.coef[(size_t)v * b2.ibass + j0 + c];
                    pdg[(size_t)v * iang1 + a] = rad * s;
                }
            // offdg += pdg^T coef1(i0 ...)
            for (int v1 = 0; v1 < mvib1; ++v1)
                for (int v2 = 0; v2 < mvib2; ++v2) {
                    double s = 0.0;
                    for (int a = 0; a < iang1; ++a)
                        s += pdg[(size_t)v2 * iang1 + a] * b1.coef[(size_t)v1 * b1.ibass + i0 + a];
                    offdg[(size_t)v1 * mvib2 + v2] += s;
                }
        }
        ir1 = ir1 + iq1;
        ir2 = ir2 + iq2;
    }
}

// dstore :1917-2049 (itra = 1): the eigenvectors transformed to the first-step basis with the
// angular DVR taken back to associated Legendre functions (tofbr :2175-2228, jtran :2230-2274),
// one record per k block, for DIPOLE3.
void rot_dstore(const char *kvec_path, const std::vector<int> &h, int ipar_out, const std::vector<unsigned char> &rec2,
                const std::vector<double> &rec3, const std::vector<double> &r, int jrot, int kmin, int ndvr,
                const std::vector<const RotBlock *> &bp, const std::vector<int> &mvib, const std::vector<double> &vec,
                int nbass, const std::vector<double> &ev, int nval) {
    const int nblk = (int)bp.size();
    std::vector<RotBlock> blk;
    for (auto *b : bp) blk.push_back(*b);
    std::vector<int> lmin(nblk), lbasis(nblk), nkbas(nblk);
    int nend = 0;
    for (int k = 0; k < nblk; ++k) {  // select :374-380
        lmin[k] = blk[k].k1;
        lbasis[k] = blk[k].maxleg + blk[k].lincr - blk[k].k1 + 1;
        nkbas[k] = (blk[k].ibass / blk[k].iang) * lbasis[k];
        nend += nkbas[k];
    }
    FILE *fp = std::fopen(kvec_path, "wb");
    if (!fp) fail(DVR3D_ERR_ARG);
    auto put = [&](const void *p, size_t n) {
        const int32_t m = (int32_t)n;
        std::fwrite(&m, 4, 1, fp);
        if (n) std::fwrite(p, 1, n, fp);
        std::fwrite(&m, 4, 1, fp);
    };
    const int hdr[8] = {h[0], ipar_out, h[2], h[3], h[4], jrot, kmin, nval};
    put(hdr, sizeof(hdr));
    put(rec2.data(), std::min<size_t>(rec2.size(), 56));  // zembed .. zncor (no zquad2)
    put(rec3.data(), 8 * rec3.size());
    std::vector<int> r4;
    r4.push_back(nend);
    r4.insert(r4.end(), lmin.begin(), lmin.end());
    r4.insert(r4.end(), lbasis.begin(), lbasis.end());
    r4.insert(r4.end(), nkbas.begin(), nkbas.end());
    put(r4.data(), 4 * r4.size());
    put(r.data(), 8 * r.size());
    put(&nval, 4);
    put(ev.data(), 8 * (size_t)nval);
    int mend = 0;
    for (int k = 0; k < nblk; ++k) {
        const RotBlock &B = blk[k];
        const int nang = lbasis[k], nrad = B.ibass / B.iang, mv = mvib[k];
        const int mbeg = mend;
        mend += mv;
        if (mv <= 0) continue;
        // jtran: b(j + mn*nang, l) = sum over kept angles of dvrvec(kk, mn) pleg(j, k)
        std::vector<double> b((size_t)nkbas[k] * mv, 0.0);
        for (int l = 0; l < mv; ++l) {
            const double *dv = &B.coef[(size_t)l * B.ibass];
            for (int j = 0; j < nang; ++j) {
                for (int mn = 0; mn < nrad; ++mn) {
                    double sumk = 0.0;
                    int kk = 0;
                    for (int a = 0; a < B.nang; ++a) {
                        if (B.iv[a] == 0) continue;
                        sumk += dv[kk + (size_t)mn * B.iang] * B.pleg[j + (size_t)a * ndvr];
                        ++kk;
                    }
                    b[(size_t)l * nkbas[k] + j + (size_t)mn * nang] = sumk;
                }
            }
        }
        // d = b c, c(mvib(k), nval): rows mbeg.. of the eigenvectors
        std::vector<double> d((size_t)nkbas[k] * nval, 0.0);
        for (int i = 0; i < nval; ++i)
            for (int l = 0; l < mv; ++l) {
                const double c = vec[(size_t)i * nbass + mbeg + l];
                for (int j = 0; j < nkbas[k]; ++j) d[(size_t)i * nkbas[k] + j] += b[(size_t)l * nkbas[k] + j] * c;
            }
        put(d.data(), 8 * d.size());
    }
    std::fclose(fp);
}

// dstore1 :2051-2173: the J = 1 f set is the first step's k = 1 f block itself; its records are
// copied in the layout of a J = 0 first-step file (read by DIPOLE3 as a one-block set).
// idvr: the angular point count of the last e-type block select read (vrmain's argument).
void rot_dstore1(const char *kvec_path, const std::vector<int> &h, int ipar_out, const std::vector<unsigned char> &rec2,
                 const std::vector<double> &rec3, const std::vector<double> &r, int idvr, int ndvr, int nmax,
                 const std::vector<double> &xalf, const RotBlock &B, const std::vector<double> &vecs, int nval) {
    FILE *fp = std::fopen(kvec_path, "wb");
    if (!fp) fail(DVR3D_ERR_ARG);
    auto put = [&](const void *p, size_t n) {
        const int32_t m = (int32_t)n;
        std::fwrite(&m, 4, 1, fp);
        if (n) std::fwrite(p, 1, n, fp);
        std::fwrite(&m, 4, 1, fp);
    };
    const int hdr[8] = {h[0], ipar_out, idvr, h[3], h[4], h[5], 0, nval};
    put(hdr, sizeof(hdr));
    put(rec2.data(), std::min<size_t>(rec2.size(), 56));
    put(rec3.data(), 8 * rec3.size());
    const int max2d = nmax * (nmax + 1 - 2 * ipar_out) / 2, mbass = idvr * max2d;
    const int r4[4] = {mbass, 0, idvr, mbass};
    put(r4, sizeof(r4));
    put(r.data(), 8 * r.size());
    put(xalf.data(), 8 * (size_t)std::min(idvr, (int)xalf.size()));
    const int kh[3] = {B.k1, B.maxleg, B.nang};
    put(kh, sizeof(kh));
    put(B.pleg.data(), 8 * (size_t)B.nang * ndvr);
    const int ib[2] = {B.iang, B.ibass};
    put(ib, sizeof(ib));
    put(B.iv.data(), 4 * (size_t)B.nang);
    put(&nval, 4);
    put(B.evib.data(), 8 * (size_t)nval);
    for (int l = 0; l < nval; ++l) put(&vecs[(size_t)l * B.ibass], 8 * (size_t)B.ibass);
    std::fclose(fp);
}

int rotlev3b_run(const char *deck_text, const char *wave_path, double *levels, int cap, int *nlev,
                 const char *kvec_path = nullptr, std::vector<double> *f_out = nullptr,
                 const char *kvec2_path = nullptr) {
    // deck: namelist, then the 12i5 card, title, optional ezero
    std::vector<std::string> lines;
    {
        std::string cur;
        for (const char *c = deck_text; *c; ++c) {
            if (*c == '\n') {
                lines.push_back(cur);
                cur.clear();
            } else if (*c != '\r') {
                cur += *c;
            }
        }
        if (!cur.empty()) lines.push_back(cur);
    }
    size_t li = 0;
    while (li < lines.size() && lines[li].find('/') == std::string::npos) ++li;
    ++li;
    if (li >= lines.size()) fail(DVR3D_ERR_DECK);
    auto i5 = [&](const std::string &s, int f) {
        if ((size_t)(5 * f) >= s.size()) return 0;
        std::string t = s.substr(5 * f, 5);
        size_t a = t.find_first_not_of(' ');
        return a == std::string::npos ? 0 : std::atoi(t.c_str() + a);
    };
    int nvib = i5(lines[li], 0), neval = i5(lines[li], 1), kmin = i5(lines[li], 2), ibass = i5(lines[li], 3);
    int neval2 = i5(lines[li], 4);
    int npnt = i5(lines[li], 5);
    // file
    RotFile f;
    {
        FILE *fp = std::fopen(wave_path, "rb");
        if (!fp) fail(DVR3D_ERR_ARG);
        std::fseek(fp, 0, SEEK_END);
        long n = std::ftell(fp);
        std::fseek(fp, 0, SEEK_SET);
        f.b.resize((size_t)n);
        if (n > 0 && std::fread(f.b.data(), 1, (size_t)n, fp) != (size_t)n) {
            std::fclose(fp);
            fail(DVR3D_ERR_ARG);
        }
        std::fclose(fp);
    }
    std::vector<int> h = f.ints();  // idia,ipar,ndvr,nmax,nmax,jrot,kmin0,meval,nlim (insize :155)
    if (h.size() < 9) fail(DVR3D_ERR_ARG);
    int idia = h[0], ipar = h[1], ndvr = h[2], nmax = h[3], jrot = h[5], kmin0 = h[6], meval = h[7];
    if (idia != -2 || jrot <= 0) fail(DVR3D_ERR_UNSUPPORTED);
    if (kmin != kmin0 && kmin0 != 2) fail(DVR3D_ERR_ARG);
    if (kmin > 2 || (kmin == 0 && kmin0 != 0)) fail(DVR3D_ERR_UNSUPPORTED);
    nvib = std::min(nvib, meval);  // insize :171-186
    int nblk = kmin > 0 ? jrot + 1 : jrot;
    if (neval <= 0) neval = 10;
    if (neval2 <= 0) neval2 = neval;
    npnt = std::max(ndvr, npnt);
    std::vector<unsigned char> rec2;
    {
        auto r = f.rec();
        rec2.assign(r.first, r.first + r.second);
    }
    std::vector<double> rec3(6);
    f.getrow(rec3.data(), 6);
    std::vector<double> rm2(nmax);
    f.getrow(rm2.data(), nmax);  // radint :686
    std::vector<double> rgrid(nmax);
    f.getrow(rgrid.data(), nmax);
    // select :345-382 (blocks read sequentially) and solrt's reads
    std::vector<RotBlock> blk(nblk);
    std::vector<int> mvib(nblk);
    int ipt = 0;
    // one k block of the file (ccmain :972-976, testiv :3446-3448, transr :3622-3641), with its
    // first `keep` vectors (at most)
    auto read_block = [&](RotBlock &B, int keep) {
        f.skip();  // xalf
        std::vector<int> kk = f.ints();
        B.k1 = kk[0];
        B.maxleg = kk[1];
        B.nang = kk[2];
        B.lincr = kk.size() > 3 ? kk[3] : 0;
        B.pleg.assign((size_t)ndvr * ndvr, 0.0);
        f.getrow(B.pleg.data(), B.nang * ndvr);
        std::vector<int> ib = f.ints();
        B.iang = ib[0];
        B.ibass = ib[1];
        std::vector<int> iv = f.ints();
        B.iv.assign(iv.begin(), iv.begin() + B.nang);
        B.meval = f.ints()[0];
        const int m = std::min(std::min(keep, B.ibass), B.meval);
        B.evib.resize(B.meval);
        f.getrow(B.evib.data(), B.meval);
        B.coef.assign((size_t)B.ibass * std::max(m, 1), 0.0);
        for (int i = 0; i < B.meval; ++i) {
            if (i < m) f.getrow(&B.coef[(size_t)i * B.ibass], B.ibass);
            else f.skip();
        }
        return m;
    };
    for (int ioff = 0; ioff < nblk; ++ioff) {
        mvib[ioff] = read_block(blk[ioff], nvib);
        ipt += mvib[ioff];
    }
    // KMIN = 2: the f-type k = 1 block follows the J + 1 e-type blocks (endiv :1635-1658)
    RotBlock endblk{};
    size_t endpos = 0;
    std::vector<double> endxalf(ndvr, 0.0);
    if (kmin == 2) {
        endpos = f.pos;
        {
            RotFile g;
            g.b = f.b;
            g.pos = endpos;
            g.getrow(endxalf.data(), ndvr);
        }
        read_block(endblk, nvib);
        if (endblk.k1 != 1) fail(DVR3D_ERR_ARG);
    }
    int nbass = ipt;
    if (ibass > 0 && ibass < ipt) {  // select :391-423
        std::vector<int> iv(nblk, 1);
        int p = 1;
        for (int n = 1; n <= ibass; ++n) {
            while (!(iv[p - 1] <= mvib[p - 1])) p = p + 1;
            double evibr = blk[p - 1].evib[iv[p - 1] - 1];
            int jpt = p;
            for (int j = p + 1; j <= nblk; ++j) {
                if (iv[j - 1] > mvib[j - 1]) continue;
                if (blk[j - 1].evib[iv[j - 1] - 1] >= evibr) continue;
                evibr = blk[j - 1].evib[iv[j - 1] - 1];
                jpt = j;
            }
            iv[jpt - 1] = iv[jpt - 1] + 1;
        }
        for (int i = 0; i < nblk; ++i) mvib[i] = iv[i] - 1;
        nbass = ibass;
    }
    neval = std::min(neval, nbass);
    int iang = 0;
    for (auto &B : blk) iang = std::max(iang, B.iang);
    // radint :686-694
    std::vector<double> radmee = rot_mkrad(nmax, rm2, 0, 0, 0), radmoo = rot_mkrad(nmax, rm2, 1, 0, 0),
                        radmeo = rot_mkrad(nmax, rm2, 1, 1, 0), radmoe = rot_mkrad(nmax, rm2, 1, 1, 1);
    double jjp1 = (double)(jrot * (jrot + 1));
    const double sqrt2 = 1.4142135623731;
    // The Hamiltonian of a chain of k blocks, in core (solrt :1414-1527, loadh :1296-1337): the
    // levels of each block on the diagonal, the Coriolis blocks of neighbours k, k+1 and k, k+2;
    // ip0 is the radial parity label of the first pair and alternates along the chain.
    auto build = [&](const std::vector<const RotBlock *> &B, const std::vector<int> &mv, int ip0,
                     std::vector<double> &ham, int &nb) {
        const int nk = (int)B.size();
        nb = 0;
        for (int v : mv) nb += v;
        ham.assign((size_t)nb * nb, 0.0);
        std::vector<int> ist(nk + 1, 0);
        for (int i = 0; i < nk; ++i) ist[i + 1] = ist[i] + mv[i];
        for (int i = 0; i < nk; ++i)
            for (int v = 0; v < mv[i]; ++v) ham[(size_t)(ist[i] + v) * nb + ist[i] + v] = B[i]->evib[v];
        auto place = [&](int i, int j, const std::vector<double> &offdg) {
            int p = 0;
            for (int i1 = 0; i1 < mv[i]; ++i1)
                for (int i2 = 0; i2 < mv[j]; ++i2) {
                    double x = offdg[p++];
                    ham[(size_t)(ist[j] + i2) * nb + ist[i] + i1] = x;
                    ham[(size_t)(ist[i] + i1) * nb + ist[j] + i2] = x;
                }
        };
        int ip = ip0;
        for (int ioff = 2; ioff <= nk; ++ioff) {
            const RotBlock &B1 = *B[ioff - 2], &B2 = *B[ioff - 1];
            int k1 = B1.k1;
            int mn = mv[ioff - 2] * mv[ioff - 1];
            double angfac = +std::sqrt(jjp1 - (double)(k1 * (k1 + 1))) / 2.0;
            if (k1 == 0) angfac = sqrt2 * angfac;
            RotQuad q;
            {
                int npnt2 = (npnt + 1) / 2;
                double tswalf = std::pow(2.0, k1 + k1 + 1) / (double)(k1 + 1);
                for (int i = 1; i <= k1; ++i) tswalf = tswalf * (double)i / (double)(k1 + i + 1);
                double cswalf;
                rot_jacobi(npnt, npnt2, q.xalf, q.walf, (double)k1, (double)k1, cswalf, tswalf);
                if (std::fabs((cswalf - tswalf) / tswalf) > 1.0e-8) fail(DVR3D_ERR_QUADRATURE);
                for (int i = 1; i <= npnt2; ++i) {
                    q.xalf[npnt + 1 - i] = q.xalf[i];
                    q.xalf[i] = -q.xalf[i];
                    q.walf[npnt + 1 - i] = q.walf[i];
                }
            }
            std::vector<double> angmat, offdg;
            if (mn > 0) {
                rot_angin(1, angmat, iang, q, npnt, ndvr, B1, B2, k1, angfac);
                if (ip == 0)
                    rot_solofd(offdg, radmeo, angmat, iang, nmax, 1, 1, 0, B1.iang, B2.iang, mv[ioff - 2],
                               mv[ioff - 1], B1, B2);
                else
                    rot_solofd(offdg, radmoe, angmat, iang, nmax, 1, 0, 1, B1.iang, B2.iang, mv[ioff - 2],
                               mv[ioff - 1], B1, B2);
                place(ioff - 2, ioff - 1, offdg);
            }
            if (ioff == nk) break;
            const RotBlock &B3 = *B[ioff];
            mn = mv[ioff - 2] * mv[ioff];
            if (mn > 0) {
                angfac = -std::sqrt((jjp1 - (double)((k1 + 1) * (k1 + 2))) * (jjp1 - (double)(k1 * (k1 + 1)))) / 16.0;
                if (k1 == 0) angfac = sqrt2 * angfac;
                rot_angin(2, angmat, iang, q, npnt, ndvr, B1, B3, k1, angfac);
                if (ip == 0)
                    rot_solofd(offdg, radmee, angmat, iang, nmax, 0, 0, 0, B1.iang, B3.iang, mv[ioff - 2],
                               mv[ioff], B1, B3);
                else
                    rot_solofd(offdg, radmoo, angmat, iang, nmax, 1, 0, 0, B1.iang, B3.iang, mv[ioff - 2],
                               mv[ioff], B1, B3);
                place(ioff - 2, ioff, offdg);
            }
            ip = 1 - ip;
        }
    };
    std::vector<const RotBlock *> chain;
    for (auto &B : blk) chain.push_back(&B);
    std::vector<double> ham;
    int nb = 0;
    build(chain, mvib, ipar, ham, nb);
    std::vector<double> ev(nbass);
    diag(ham.data(), nbass, nbass, ev.data());
    const int kmin_e = kmin == 2 ? 1 : kmin;
    if (kvec_path) rot_dstore(kvec_path, h, ipar, rec2, rec3, rgrid, jrot, kmin_e, ndvr, chain, mvib, ham, nbass, ev, neval);
    *nlev = neval;
    if (levels) {
        if (cap < neval) fail(DVR3D_ERR_BUFFER);
        for (int i = 0; i < neval; ++i) levels[i] = ev[i];
    }
    if (kmin == 2 && f_out) {
        // the second pass, f parity (vrmain :600-660): k = 1..J with the f-type k = 1 block stored
        // at the end of the first-step file; the Coriolis blocks among k >= 2 are the first
        // pass's, those of the k = 1 f block are formed anew (solrt :1529-1617), ip = 1 - ipar
        const int nbf = nbass - mvib[0];
        int nevf = std::min(neval2, nbf);
        std::vector<double> evf;
        if (jrot == 1) {
            // J = 1 f: the k = 1 f block alone (dstore1 :2051-2173)
            nevf = std::min(nevf, endblk.meval);
            evf.assign(endblk.evib.begin(), endblk.evib.begin() + nevf);
            if (kvec2_path) {
                RotBlock e1 = endblk;
                std::vector<double> vecs;
                // all nevf vectors of the block, re-read (the e pass kept at most nvib)
                RotFile g;
                g.b = f.b;
                g.pos = endpos;
                g.skip();
                g.skip();
                g.skip();
                g.skip();
                g.skip();
                g.skip();
                g.skip();
                vecs.assign((size_t)e1.ibass * nevf, 0.0);
                for (int l = 0; l < nevf; ++l) g.getrow(&vecs[(size_t)l * e1.ibass], e1.ibass);
                rot_dstore1(kvec2_path, h, 1 - ipar, rec2, rec3, rgrid, blk[nblk - 1].nang, ndvr, nmax, endxalf, e1, vecs,
                            nevf);
            }
        } else {
            std::vector<const RotBlock *> fchain{&endblk};
            std::vector<int> mvf{mvib[1]};
            for (int i = 2; i < nblk; ++i) {
                fchain.push_back(&blk[i]);
                mvf.push_back(mvib[i]);
            }
            if (mvf[0] > (int)endblk.evib.size() || (size_t)mvf[0] * endblk.ibass > endblk.coef.size())
                fail(DVR3D_ERR_ARG);
            std::vector<double> hf;
            int nbf2 = 0;
            build(fchain, mvf, 1 - ipar, hf, nbf2);
            if (nbf2 != nbf) fail(DVR3D_ERR_ARG);
            evf.assign(nbf, 0.0);
            diag(hf.data(), nbf, nbf, evf.data());
            // the f k = 1 block takes the e-type k = 1 block's place in the labels (select
            // :374-380 ran on the e blocks); the two must agree in size
            const int nk1e = (blk[1].ibass / blk[1].iang) * (blk[1].maxleg + blk[1].lincr - blk[1].k1 + 1);
            const int nk1f = (endblk.ibass / endblk.iang) * (endblk.maxleg + endblk.lincr - endblk.k1 + 1);
            if (kvec2_path && nk1e != nk1f) fail(DVR3D_ERR_UNSUPPORTED);
            if (kvec2_path)
                rot_dstore(kvec2_path, h, 1 - ipar, rec2, rec3, rgrid, jrot, 0, ndvr, fchain, mvf, hf, nbf, evf, nevf);
            evf.resize(nevf);
        }
        *f_out = evf;
    }
    return DVR3D_OK;
}

}  // namespace

extern "C" {

int oracle_dsyev_lower(double *a, int n, double *w) {
    try {
        diag(a, n, n, w);
        return DVR3D_OK;
    } catch (const Fail &f) {
        return f.code;
    }
}

int oracle_load_lapack(const char *path, const char *prefix) {
    void *h = dlopen(path, RTLD_NOW | RTLD_LOCAL);
    if (!h) return DVR3D_ERR_ARG;
    std::string p(prefix ? prefix : "");
    g_dsyev = (dsyev_t)dlsym(h, (p + "dsyev_").c_str());
    g_dsyevd = (dsyevd_t)dlsym(h, (p + "dsyevd_").c_str());
    return g_dsyev ? DVR3D_OK : DVR3D_ERR_ARG;
}

double oracle_pes_morse_sum(const double *p, double r1, double r2, double xcos) {
    return pes_morse_sum(p, r1, r2, xcos);
}

int oracle_sizes(const dvr3d_deck *deck, int kk, int *o) {
    try {
        Run R;
        insize_setcon(R, *deck);
        ccmain_setup(R, kk);
        int v[16] = {R.npnt1, R.npnt2, R.nalf, R.idvr, R.npnta, R.npntb, R.npntc, R.max2d,
                     R.max3d, R.neval, R.kz, R.ipar, R.nidvr, R.lincr, R.kd, R.ku};
        std::memcpy(o, v, sizeof(v));
        return DVR3D_OK;
    } catch (Fail &f) {
        return f.code;
    }
}

int oracle_quadrature(const dvr3d_deck *deck, int kk, oracle_quad *q) {
    std::memset(q, 0, sizeof(*q));
    Run R;
    int status = DVR3D_OK;
    try {
        insize_setcon(R, *deck);
        ccmain_setup(R, kk);
    } catch (Fail &f) {
        status = f.code;
    }
    q->status = status;
    q->npnt1 = (int)R.y1.size();
    q->npnt2 = (int)R.y2.size();
    for (size_t i = 0; i < R.y1.size() && i < 128; ++i) {
        q->y1[i] = R.y1[i];
        q->wt1[i] = R.wt1[i];
        q->r1[i] = R.r1.size() > i ? R.r1[i] : 0.0;
    }
    for (size_t i = 0; i < R.y2.size() && i < 128; ++i) {
        q->y2[i] = R.y2[i];
        q->wt2[i] = R.wt2[i];
        q->r2[i] = R.r2.size() > i ? R.r2[i] : 0.0;
    }
    q->csx1 = R.csx1; q->csa1 = R.csa1; q->tsx1 = R.tsx1; q->tsa1 = R.tsa1;
    q->csx2 = R.csx2; q->csa2 = R.csa2; q->tsx2 = R.tsx2; q->tsa2 = R.tsa2;
    q->nang2 = (int)R.xhalf.size();
    for (size_t i = 0; i < R.xhalf.size() && i < 128; ++i) {
        q->xhalf[i] = R.xhalf[i];
        q->whalf[i] = R.whalf[i];
    }
    q->cswalf = R.cswalf;
    q->tswalf = R.tswalf;
    q->nidvr = (int)R.xalf.size();
    for (size_t i = 0; i < R.xalf.size() && i < 256; ++i) {
        q->xalf[i] = R.xalf[i];
        q->walf[i] = R.walf[i];
    }
    q->ur1 = R.ur1; q->ur2 = R.ur2; q->urr1 = R.urr1; q->urr2 = R.urr2;
    q->beta1 = R.beta1; q->beta2 = R.beta2; q->a1 = R.a1; q->a2 = R.a2;
    q->g1 = R.g1; q->g2 = R.g2; q->iu1 = R.iu1; q->iu2 = R.iu2;
    return status;
}

int oracle_solve_block(const dvr3d_deck *deck, int kk, int pes_kind, const double *pes,
                       int npes, const double *vgrid, size_t nvgrid, int final_mode,
                       oracle_trace *trace, dvr3d_result *res) {
    try {
        Run R;
        insize_setcon(R, *deck);
        R.pes_kind = pes_kind;
        if (pes_kind == DVR3D_PES_MORSE_SUM) {
            if (!pes || npes < DVR3D_PES_MORSE_SUM_NPARAM) return DVR3D_ERR_ARG;
            R.pes.assign(pes, pes + DVR3D_PES_MORSE_SUM_NPARAM);
        }
        R.vgrid = vgrid;
        R.nvgrid = nvgrid;
        ccmain_setup(R, kk);
        if (trace) {
            trace->npnta = R.npnta;
            trace->npntb = R.npntb;
            trace->npntc = R.npntc;
            trace->max2d = R.max2d;
            trace->max3d = R.max3d;
            trace->kz = R.kz;
            trace->ipar = R.ipar;
        }
        if (R.idia <= -2) nfmain(R, final_mode, trace, res);
        else jhmain(R, final_mode, trace, res);
        return DVR3D_OK;
    } catch (Fail &f) {
        return f.code;
    } catch (std::exception &) {
        return DVR3D_ERR_NOMEM;
    }
}

// ------------------------------------------------------------------ stepwise runs
// One k-block solve executed on a worker thread in units of work, so a caller can time one
// complete solve as a sequence of bounded steps: each oracle_session_step call lets the
// worker run the next `units` units (gates of nfmain / jhmain) and returns when they are
// done. The worker is blocked between steps.
struct OracleSession {
    Run R;
    int final_mode = 0;
    int units = 0;
    std::thread worker;
    std::mutex mu;
    std::condition_variable cv;
    long long granted = 0, passed = 0;
    bool blocked = false, finished = false, cancel = false;
    int status = 0;
    std::vector<double> eval;
    std::vector<int> iv2;
    oracle_trace tr{};
    dvr3d_result res{};
};

struct Cancelled {};

int oracle_session_begin(const dvr3d_deck *deck, int kk, int pes_kind, const double *pes, int npes,
                         const double *vgrid, size_t nvgrid, int final_mode, void **out) {
    if (!deck || !out) return DVR3D_ERR_ARG;
    auto *S = new OracleSession();
    try {
        Run &R = S->R;
        insize_setcon(R, *deck);
        R.pes_kind = pes_kind;
        if (pes_kind == DVR3D_PES_MORSE_SUM) {
            if (!pes || npes < DVR3D_PES_MORSE_SUM_NPARAM) {
                delete S;
                return DVR3D_ERR_ARG;
            }
            R.pes.assign(pes, pes + DVR3D_PES_MORSE_SUM_NPARAM);
        }
        R.vgrid = vgrid;
        R.nvgrid = nvgrid;
        ccmain_setup(R, kk);
    } catch (Fail &f) {
        delete S;
        return f.code;
    }
    S->final_mode = final_mode;
    S->units = work_units(S->R);
    S->eval.assign(std::max(S->R.neval, 1), 0.0);
    S->iv2.assign(std::max(std::max(S->R.nalf, S->R.npntc), 1), 0);
    S->res.eval = S->eval.data();
    S->res.eval_cap = (int)S->eval.size();
    S->tr.iv2 = S->iv2.data();
    S->tr.iv2_cap = (int)S->iv2.size();
    S->R.gate = [S]() {
        std::unique_lock<std::mutex> lk(S->mu);
        S->blocked = true;
        S->cv.notify_all();
        S->cv.wait(lk, [S] { return S->cancel || S->passed < S->granted; });
        S->blocked = false;
        if (S->cancel) throw Cancelled{};
        ++S->passed;
    };
    S->worker = std::thread([S]() {
        int st = DVR3D_OK;
        try {
            if (S->R.idia <= -2) nfmain(S->R, S->final_mode, &S->tr, &S->res);
            else jhmain(S->R, S->final_mode, &S->tr, &S->res);
        } catch (Fail &f) {
            st = f.code;
        } catch (Cancelled &) {
            st = DVR3D_ERR_ARG;
        } catch (std::exception &) {
            st = DVR3D_ERR_NOMEM;
        }
        std::lock_guard<std::mutex> lk(S->mu);
        S->status = st;
        S->finished = true;
        S->cv.notify_all();
    });
    *out = S;
    return DVR3D_OK;
}

int oracle_session_units(void *h) { return h ? static_cast<OracleSession *>(h)->units : DVR3D_ERR_ARG; }

int oracle_session_counts(void *h, int *iv2, int *n2d, int cap) {
    if (!h) return DVR3D_ERR_ARG;
    auto *S = static_cast<OracleSession *>(h);
    std::lock_guard<std::mutex> lk(S->mu);
    if (!(S->blocked || S->finished)) return DVR3D_ERR_ARG;  // only between steps
    const int nb = (int)S->R.sel_iv2.size();
    if (nb == 0) return 0;  // the selection has not run yet
    if (cap < nb) return DVR3D_ERR_BUFFER;
    for (int b = 0; b < nb; ++b) {
        if (iv2) iv2[b] = S->R.sel_iv2[b];
        if (n2d) n2d[b] = S->R.sel_n2d[b];
    }
    return nb;
}

int oracle_session_step(void *h, int units) {
    if (!h || units < 0) return DVR3D_ERR_ARG;
    auto *S = static_cast<OracleSession *>(h);
    std::unique_lock<std::mutex> lk(S->mu);
    S->granted += units;
    S->cv.notify_all();
    // done when the worker waits at the gate after the granted units, or has finished
    S->cv.wait(lk, [S] { return S->finished || (S->blocked && S->passed == S->granted); });
    if (S->finished && S->status != DVR3D_OK) return S->status;
    return S->finished ? 0 : (int)(S->units - S->passed);
}

int oracle_session_end(void *h, oracle_trace *trace, dvr3d_result *res) {
    if (!h) return DVR3D_ERR_ARG;
    auto *S = static_cast<OracleSession *>(h);
    {
        std::lock_guard<std::mutex> lk(S->mu);
        if (!S->finished) S->cancel = true;
        S->cv.notify_all();
    }
    S->worker.join();
    const int st = S->status;
    if (st == DVR3D_OK) {
        if (res) {
            res->nham3 = S->res.nham3;
            res->meval = S->res.meval;
            res->nblocks = S->res.nblocks;
            res->kz = S->res.kz;
            res->ipar = S->res.ipar;
            if (res->eval && res->eval_cap >= S->res.meval)
                std::memcpy(res->eval, S->eval.data(), sizeof(double) * S->res.meval);
        }
        if (trace) {
            trace->nblocks = S->tr.nblocks;
            trace->nham3 = S->tr.nham3;
            std::memcpy(trace->stage_s, S->tr.stage_s, sizeof(trace->stage_s));
            if (trace->iv2 && trace->iv2_cap >= S->tr.nblocks)
                std::memcpy(trace->iv2, S->iv2.data(), sizeof(int) * S->tr.nblocks);
        }
    }
    delete S;
    return st;
}

double oracle_time_dsyev(int n, int reps, int mode) {
    std::mt19937_64 rng(12345);
    std::uniform_real_distribution<double> u(-1.0, 1.0);
    std::vector<double> a0((size_t)n * n), a((size_t)n * n), w(n);
    for (int j = 0; j < n; ++j)
        for (int i = j; i < n; ++i) a0[(size_t)j * n + i] = a0[(size_t)i * n + j] = u(rng);
    double tot = 0.0;
    for (int r = 0; r < reps; ++r) {
        a = a0;
        auto t0 = std::chrono::steady_clock::now();
        try {
            diag(a.data(), n, n, w.data(), mode);
        } catch (Fail &) {
            return -1.0;
        }
        tot += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    return tot / reps;
}

int oracle_rot_quadrature(int npnt, int k, double *x, double *w, double *cswalf, double *tswalf) {
    try {
        int npnt2 = (npnt + 1) / 2;
        double ts = std::pow(2.0, k + k + 1) / (double)(k + 1);
        for (int i = 1; i <= k; ++i) ts = ts * (double)i / (double)(k + i + 1);
        std::vector<double> xa, wa;
        double cs = 0.0;
        rot_jacobi(npnt, npnt2, xa, wa, (double)k, (double)k, cs, ts);
        for (int i = 1; i <= npnt2; ++i) {
            x[i - 1] = xa[i];
            w[i - 1] = wa[i];
        }
        *cswalf = cs;
        *tswalf = ts;
        return DVR3D_OK;
    } catch (Fail &f) {
        return f.code;
    }
}

int oracle_rotlev3b(const char *deck_text, const char *wave_path, double *levels, int cap, int *nlev) {
    if (!deck_text || !wave_path || !nlev) return DVR3D_ERR_ARG;
    try {
        return rotlev3b_run(deck_text, wave_path, levels, cap, nlev);
    } catch (Fail &f) {
        return f.code;
    }
}

int oracle_rotlev3b_pair(const char *deck_text, const char *wave_path, const char *kvec_path, const char *kvec2_path,
                         double *levels, int cap, int *nlev, double *levels2, int cap2, int *nlev2) {
    if (!deck_text || !wave_path || !nlev || !nlev2) return DVR3D_ERR_ARG;
    try {
        std::vector<double> f;
        int rc = rotlev3b_run(deck_text, wave_path, levels, cap, nlev, (kvec_path && kvec_path[0]) ? kvec_path : nullptr,
                              &f, (kvec2_path && kvec2_path[0]) ? kvec2_path : nullptr);
        if (rc != DVR3D_OK) return rc;
        *nlev2 = (int)f.size();
        if (levels2) {
            if (cap2 < (int)f.size()) return DVR3D_ERR_BUFFER;
            for (size_t i = 0; i < f.size(); ++i) levels2[i] = f[i];
        }
        return DVR3D_OK;
    } catch (Fail &e) {
        return e.code;
    }
}

int oracle_rotlev3b_trans(const char *deck_text, const char *wave_path, const char *kvec_path, double *levels,
                          int cap, int *nlev) {
    if (!deck_text || !wave_path || !kvec_path || !nlev) return DVR3D_ERR_ARG;
    try {
        return rotlev3b_run(deck_text, wave_path, levels, cap, nlev, kvec_path);
    } catch (Fail &f) {
        return f.code;
    }
}

}  // extern "C"
