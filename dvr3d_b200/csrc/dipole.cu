// dipole.cu -- transition moments between the vib-rot states of two wavefunction files: the
// reference's program DIPOLE3 (source/dipole3_segmented.f90), with its contractions on the GPU.
//
// For every k -> k' block the reference evaluates the states of both files at the angular
// integration points (dsrd :1412-1562; for a J = 0 first-step file the angular DVR is first taken
// back to associated Legendre functions, jtran :1564-1646) and sums
//     t(i1, i2) += x1 * dipol(p) * psi1(i1, p) * psi2(i2, p)   over the points p
// with one rank-1 update per point (trans :1648-1776). Here
//   * the angular DVR -> FBR transform of a J = 0 file is one GEMM over all radial functions and
//     states (FBR (nang x nrad ne) = P'' (nang x iang) V (iang x nrad ne));
//   * the Legendre functions at the points: A (ipot x nrad ne) = Pd (ipot x nang) FBR;
//   * trans: T (ne1 x ne2) += A1^T diag(x1 w dipol) A2, the diagonal folded into A2 by one
//     kernel, then one GEMM with K = nrad ipot.
// All three are FP64 tensor-core (DMMA) GEMMs of gemm64. The host reads and checks the two files
// (insize :198-620, genind :656-706), packs each block's vectors as the reference indexes them
// (symmetric radial points dropped where dsrd / jtran drop them), calls the user's dipole
// plug-in at the points (lagpt :1141-1232, DIPD :2054-2194) and prints spect's table (:1825-1954)
// and writes outpt's records (:1956-2003).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/dvr3d_b200.h"
#include "common.cuh"
#include "dipole.cuh"
#include "gemm64.cuh"
#include "pipeline.cuh"
#include "wavefile.cuh"

#define CK(x)                                          \
    do {                                               \
        cudaError_t e_ = (x);                          \
        if (e_ != cudaSuccess) throw CudaFail{e_, #x}; \
    } while (0)

namespace dvr3d {

namespace {

[[noreturn]] void bad(int code, const std::string &m) { throw HostError{code, m}; }

// ---- the job deck: namelist PRT, title (9a8), NPOT NV1 NV2 IBASE1 IBASE2 (5i5), EZERO (f20.0)
struct DipCards {
    bool zpmin = false, ztra = true, zstart = false;  // block data :180-186
    int ires = 0, nblock = 1000;
    std::string title;
    int npot = 0, nv1 = 0, nv2 = 0, ibase1 = 0, ibase2 = 0;
    bool have_ezero = false;
    double ezero = 0.0;
};

DipCards read_cards(const char *text) {
    std::vector<std::string> ln(1);
    for (const char *c = text; *c; ++c) {
        if (*c == '\n') ln.emplace_back();
        else if (*c != '\r') ln.back() += *c;
    }
    if (ln.back().empty()) ln.pop_back();
    size_t i = 0;
    while (i < ln.size() && ln[i].find('&') == std::string::npos) ++i;
    if (i == ln.size()) bad(DVR3D_ERR_DECK, "DIPOLE3 deck: no namelist PRT");
    std::string nl;
    for (; i < ln.size(); ++i) {
        nl += ln[i] + ' ';
        if (ln[i].find('/') != std::string::npos) break;
    }
    if (i == ln.size()) bad(DVR3D_ERR_DECK, "DIPOLE3 deck: namelist PRT not closed by '/'");
    ++i;
    for (auto &c : nl) c = (char)std::tolower((unsigned char)c);
    nl = nl.substr(nl.find('&') + 1);
    nl = nl.substr(0, nl.find('/'));
    // tokens: the group name, then key = value pairs separated by blanks or commas
    std::vector<std::string> tok;
    std::string cur;
    for (char c : nl) {
        if (c == ' ' || c == ',' || c == '\t' || c == '=') {
            if (!cur.empty()) tok.push_back(cur);
            cur.clear();
            if (c == '=') tok.push_back("=");
        } else {
            cur += c;
        }
    }
    if (!cur.empty()) tok.push_back(cur);
    DipCards d;
    for (size_t t = 1; t + 2 < tok.size(); ++t) {
        if (tok[t + 1] != "=") continue;
        const std::string &k = tok[t], &v = tok[t + 2];
        const bool on = (v[0] == '.' ? v.size() > 1 && v[1] == 't' : v[0] == 't');
        if (k == "zpmin") d.zpmin = on;
        else if (k == "ztra") d.ztra = on;
        else if (k == "zstart") d.zstart = on;
        else if (k == "ires") d.ires = std::atoi(v.c_str());
        else if (k == "nblock") d.nblock = std::atoi(v.c_str());
        t += 2;
    }
    if (i < ln.size()) d.title = ln[i++].substr(0, 72);
    if (i >= ln.size()) bad(DVR3D_ERR_DECK, "DIPOLE3 deck: no NPOT card");
    auto f5 = [&](int f) {
        const std::string &s = ln[i];
        if ((size_t)(5 * f) >= s.size()) return 0;
        const std::string t = s.substr(5 * f, 5);
        const size_t a = t.find_first_not_of(' ');
        return a == std::string::npos ? 0 : std::atoi(t.c_str() + a);
    };
    d.npot = f5(0);
    d.nv1 = f5(1);
    d.nv2 = f5(2);
    d.ibase1 = f5(3);
    d.ibase2 = f5(4);
    ++i;
    if (i < ln.size()) {
        std::string t = ln[i].substr(0, std::min<size_t>(20, ln[i].size()));
        for (auto &c : t)
            if (c == 'd' || c == 'D') c = 'e';
        d.have_ezero = true;
        if (t.find_first_not_of(' ') != std::string::npos) {
            char *end = nullptr;
            d.ezero = std::strtod(t.c_str(), &end);
            if (end == t.c_str()) bad(DVR3D_ERR_DECK, "DIPOLE3 deck: EZERO card is not a number");
        }
    }
    return d;
}

// ---- one wavefunction file and its header records
struct Wave {
    Records f;
    int idia = 0, ipar = 0, lmax = 0, nmax1 = 0, nmax2 = 0, jrot = 0, kmin = 0, neval = 0;
    bool zemb = false, zmor1 = false, zmor2 = false, znco = false;
    double xm[3] = {}, g1 = 0.0, g2 = 0.0, morse[6] = {};
    explicit Wave(const char *path) : f(path) {
        const std::vector<int> h = f.ints(8);
        idia = h[0];
        ipar = h[1];
        lmax = h[2];
        nmax1 = h[3];
        nmax2 = h[4];
        jrot = h[5];
        kmin = h[6];
        neval = h[7];
        const auto r = f.take();
        if (r.second < 56) bad(DVR3D_ERR_ARG, "wavefunction file: short flags record");
        auto l4 = [&](int o) {
            int32_t v;
            std::memcpy(&v, r.first + o, 4);
            return v != 0;
        };
        zemb = l4(0);
        zmor1 = l4(4);
        zmor2 = l4(8);
        std::memcpy(xm, r.first + 12, 24);
        std::memcpy(&g1, r.first + 36, 8);
        std::memcpy(&g2, r.first + 44, 8);
        znco = l4(52);
        const std::vector<double> m = f.dbls(6);
        std::copy(m.begin(), m.begin() + 6, morse);
    }
};

// ---- the dipole at the points: the user's DIPD, or the reference's DIPD around DIPSA
struct DipoleFn {
    dvr3d_dipd_fn dipd;
    dvr3d_dipsa_fn dipsa;
    void *user;
    double g1, g2;
    bool zembed, zbisc;

    double operator()(double r1, double r2, double xcos, int nu) const {
        const double v = dipd ? dipd(r1, r2, xcos, nu, user) : via_dipsa(r1, r2, xcos, nu);
        if (!std::isfinite(v)) bad(DVR3D_ERR_ARG, "dipole plug-in returned a non-finite value");
        return v;
    }

    // DIPD (:2054-2194): generalised coordinates -> bond lengths q1, q2 and angle, DIPSA's
    // bond-frame components rotated into the embedding frame of the wavefunctions.
    double via_dipsa(double r1, double r2, double xc, int nu) const {
        const double tiny = 9.0e-15;
        double q1, q2, cth, th, bet = 0.0, alf = 0.0;
        const int kind = g1 == 0.0 ? 0 : (g2 == 0.0 ? 1 : 2);  // bond-angle, scattering, general
        if (kind == 0) {
            q1 = r1;
            q2 = r2;
            cth = xc;
            th = std::acos(xc);
        } else if (kind == 1) {
            const double a = r1 * g1, b = r1 * (1.0 - g1);
            alf = std::acos(xc);
            if (r2 == 0.0 || xc >= 1.0 - tiny) {
                q1 = std::fabs(a - r2);
                q2 = b + r2;
                cth = -1.0;
            } else if (xc <= tiny - 1.0) {
                q1 = a + r2;
                q2 = std::fabs(b + r2);
                cth = 1.0;
            } else {
                q1 = std::sqrt(a * a + r2 * r2 - 2.0 * a * r2 * xc);
                q2 = std::sqrt(b * b + r2 * r2 + 2.0 * b * r2 * xc);
                cth = (q1 * q1 + q2 * q2 - r1 * r1) / (2.0 * q1 * q2);
            }
            th = std::acos(cth);
            bet = std::asin(std::sqrt(1.0 - xc * xc) * b / q2);
        } else {
            const double f1 = 1.0 / g1, f2 = 1.0 / g2, f12 = 1.0 - f1 * f2;
            const double p1 = r1 * (1.0 - f1) / (g2 * f12), p2 = r2 * (1.0 - f2) / (g1 * f12);
            const double s1 = r1 - p1, s2 = r2 - p2;
            q1 = std::sqrt(p1 * p1 + s2 * s2 + 2.0 * p1 * s2 * xc) / (1.0 - g1);
            q2 = std::sqrt(p2 * p2 + s1 * s1 + 2.0 * p2 * s1 * xc) / (1.0 - g2);
            const double q3 = std::sqrt(p1 * p1 + p2 * p2 - 2.0 * p1 * p2 * xc);
            cth = (q1 * q1 + q2 * q2 - q3 * q3) / (2.0 * q1 * q2);
            th = std::acos(cth);
        }
        double dx = 0.0, dy = 0.0;
        dipsa(&dx, &dy, q1, q2, cth, user);
        if (kind == 0) {
            const double c = std::cos(th / 2.0), s = std::sin(th / 2.0);
            if (zembed) return nu == 0 ? dy * c - dx * s : dx * c + dy * s;
            return nu == 0 ? dy * c + dx * s : -dx * c + dy * s;
        }
        if (kind == 1) {
            const double gam = bet - th / 2.0;
            if (zembed) {
                const double c = std::cos(gam), s = std::sin(gam);
                return nu == 0 ? -dx * s - dy * c : dx * c - dy * s;
            }
            const double c = std::cos(alf - gam), s = std::sin(alf - gam);
            return nu == 0 ? dx * s + dy * c : dx * c - dy * s;
        }
        if (zbisc) {
            const double h1 = g1 * q1;
            const double ca = (r2 * r2 + q2 * q2 - h1 * h1) / (2.0 * r2 * q2);
            const double a = (std::acos(xc) - th) / 2.0 - std::acos(ca);
            const double c = -std::cos(a), s = std::sin(a);
            return nu == 1 ? dx * s - dy * c : -dx * c - dy * s;
        }
        if (zembed) {
            const double h1 = g1 * q1;
            const double a = std::acos((r2 * r2 + h1 * h1 - q2 * q2) / (2.0 * r2 * h1));
            const double c = -std::cos(a + th / 2.0), s = std::sin(a + th / 2.0);
            return nu == 0 ? -dx * s + dy * c : dx * c + dy * s;
        }
        const double h2 = g2 * q2;
        const double a = std::acos((r1 * r1 + h2 * h2 - q1 * q1) / (2.0 * r1 * h2));
        const double c = -std::cos(a + th / 2.0), s = std::sin(a + th / 2.0);
        return nu == 0 ? dx * s + dy * c : -dx * c + dy * s;
    }
};

// Gauss-Legendre rule of lagpt: jacobi (:1311-1368) with alf = bta = 0, Stroud and Secrest's
// starting values refined by Newton (root :1370-1387, recur :1389-1410). Returns the nn/2
// largest points (descending) and weights, the computed and the exact half sums.
void legendre_half(int nn, std::vector<double> &x, std::vector<double> &w, double &csa, double &tsa) {
    std::vector<double> c(nn + 1, 0.0);
    for (int i = 2; i <= nn; ++i) {
        const double t = (double)i;
        c[i] = 4.0 * (t - 1.0) * (t - 1.0) * (t - 1.0) * (t - 1.0) /
               ((2.0 * t - 1.0) * (2.0 * t - 2.0) * (2.0 * t - 2.0) * (2.0 * t - 3.0));
    }
    double cc = 2.0;  // beta 2^(alf + bta + 1)
    tsa = cc / 2.0;
    for (int i = 2; i <= nn; ++i) cc *= c[i];
    auto evalp = [&](double z, double &p, double &dp, double &p1) {
        double pa = 1.0, pb = z, da = 0.0, db = 1.0;
        for (int j = 2; j <= nn; ++j) {
            const double q = z * pb - c[j] * pa, dq = z * db + pb - c[j] * da;
            pa = pb;
            pb = q;
            da = db;
            db = dq;
        }
        p = pb;
        dp = db;
        p1 = pa;
    };
    const int n2 = nn / 2;
    const double fn = nn;
    x.assign(n2 + 1, 0.0);
    w.assign(n2 + 1, 0.0);
    csa = 0.0;
    double z = 0.0;
    for (int i = 1; i <= n2; ++i) {
        if (i == 1) z = 1.0 - (2.78 / (4.0 + fn * fn)) / 1.0;
        else if (i == 2) z = z - 4.1 * (1.0 + 0.06 * (fn - 8.0) / fn) * (1.0 - z);
        else if (i == 3) z = z - 1.67 * (1.0 + 0.22 * (fn - 8.0) / fn) * (x[1] - z);
        else z = 3.0 * x[i - 1] - 3.0 * x[i - 2] + x[i - 3];
        double p = 0, dp = 1, p1 = 0;
        for (int it = 1;; ++it) {
            evalp(z, p, dp, p1);
            const double d = p / dp;
            z -= d;
            if (!(std::fabs(d) > 1.0e-12 && it < 10)) break;
        }
        x[i] = z;
        w[i] = cc / (dp * p1);
        csa += w[i];
    }
}

// Normalised associated Legendre functions P_l^m, l = m .. m + lmax, at the points, with the
// sin^m factor (asleg :1234-1309): P (npt x (lmax + 1)), column-major.
std::vector<double> legendre_at(const std::vector<double> &x, int lmax, int m) {
    const int n = (int)x.size();
    std::vector<double> P((size_t)n * (lmax + 2), 0.0);
    for (int i = 0; i < n; ++i) {
        if (std::fabs(x[i]) > 1.0) bad(DVR3D_ERR_ARG, "angular point outside [-1, 1]");
        const double s = std::sqrt((1.0 - x[i]) * (1.0 + x[i]));
        double pm = 1.0, f = 1.0;
        for (int j = 0; j < m; ++j) {
            pm = -pm * f * s;
            f += 2.0;
        }
        double pm1 = x[i] * (2 * m + 1) * pm;
        P[i] = pm;
        P[(size_t)n + i] = pm1;
        for (int l = m + 2, col = 2; l <= lmax + m; ++l, ++col) {
            const double pl = (x[i] * (2 * l - 1) * pm1 - (l + m - 1) * pm) / (double)(l - m);
            pm = pm1;
            pm1 = pl;
            P[(size_t)col * n + i] = pl;
        }
    }
    for (int j = m, col = 0; j <= lmax + m; ++j, ++col) {
        double f = 1.0;
        for (int i = j - m + 1; i <= j + m; ++i) f *= (double)i;
        const double nrm = std::sqrt((double)(2 * j + 1) / (f + f));
        for (int i = 0; i < n; ++i) P[(size_t)col * n + i] *= nrm;
    }
    return P;
}

// Wigner 3j symbol by Racah's sum over binomial coefficients (threej :1778-1823, setfac
// :1118-1139).
double wigner3j(int j1, int j2, int j3, int m1, int m2, int m3) {
    if (m1 + m2 + m3 != 0) return 0.0;
    const int a = -j1 + j2 + j3, b = j1 - j2 + j3, c = j1 + j2 - j3;
    if (a < 0 || b < 0 || c < 0 || j1 + m1 < 0 || j2 + m2 < 0 || j3 + m3 < 0 || j1 - m1 < 0 || j2 - m2 < 0 ||
        j3 - m3 < 0)
        return 0.0;
    const int nb = j1 + j2 + j3 + 3;
    std::vector<double> B((size_t)nb * nb, 0.0);  // B[i][j] = C(i, j)
    for (int i = 0; i < nb; ++i) {
        B[(size_t)i * nb] = 1.0;
        for (int j = 1; j <= i; ++j) B[(size_t)i * nb + j] = B[(size_t)(i - 1) * nb + j - 1] + (j < i ? B[(size_t)(i - 1) * nb + j] : 0.0);
    }
    auto C = [&](int n, int k) { return (k < 0 || k > n) ? 0.0 : B[(size_t)n * nb + k]; };
    const int n1 = -j1 - m2 + j3, n2 = m1 - j2 + j3, n3 = j1 - j2 + m3;
    const int kmin = std::max({-n1, -n2, 0}), kmax = std::min({j1 - m1, j2 + m2, c});
    if (kmin > kmax) return 0.0;
    double s = 0.0, sg = 1.0;
    for (int k = kmin; k <= kmax; ++k) {
        sg = -sg;
        s += sg * C(a, n1 + k) * C(b, n2 + k) * C(c, k);
    }
    s *= std::sqrt(C(2 * j2, c) * C(2 * j1, b) /
                   (C(j1 + j2 + j3 + 1, c) * (double)(2 * j3 + 1) * C(2 * j1, j1 - m1) * C(2 * j2, j2 - m2) *
                    C(2 * j3, j3 - m3)));
    // the reference's sign runs from -1 at its first term (imin = kmin + 1)
    if ((n3 + kmin + 1) % 2 != 0) s = -s;
    return s;
}

// A (K x n) rows scaled: out(p, l) = w(p) A(p, l)
__global__ void scale_rows_kernel(const double *A, long long lda, const double *w, int K, int n, double *out) {
    const long long tot = (long long)K * n;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += (long long)gridDim.x * blockDim.x) {
        const int p = (int)(t % K);
        const long long l = t / K;
        out[t] = w[p] * A[p + l * lda];
    }
}

unsigned grid_for(long long n) { return (unsigned)std::min<long long>((n + 255) / 256, 4096); }

std::string fortran_e(double v, int w, int d, char e) {  // Ew.d / Dw.d: 0.ddddE+xx
    char buf[64];
    if (v == 0.0) {
        std::snprintf(buf, sizeof(buf), "0.%0*d%c+00", d, 0, e);
    } else {
        int ex = (int)std::floor(std::log10(std::fabs(v))) + 1;
        const double sc = std::pow(10.0, d);
        double m = std::round(std::fabs(v) / std::pow(10.0, ex) * sc);
        if (m >= sc) {
            m /= 10.0;
            ++ex;
        }
        if (m < sc / 10.0) {
            m *= 10.0;
            --ex;
        }
        std::snprintf(buf, sizeof(buf), "%s0.%0*.0f%c%c%02d", v < 0 ? "-" : "", d, m, e, ex < 0 ? '-' : '+', std::abs(ex));
    }
    std::string s(buf);
    return (int)s.size() < w ? std::string(w - s.size(), ' ') + s : s;
}

std::string fortran_es(double v, int w, int d) {  // ESw.d
    char buf[64];
    std::snprintf(buf, sizeof(buf), "%.*E", d, v);
    std::string s(buf);
    return (int)s.size() < w ? std::string(w - s.size(), ' ') + s : s;
}

struct Dip {
    dvr3d_ctx *ctx;
    cudaStream_t st;
    DipCards cd;
    Wave *W[2];
    int idia = 0, ipar[2] = {}, jrot[2] = {}, kmin[2] = {}, jk[2] = {}, mbass[2] = {}, ne[2] = {}, ibase[2] = {};
    int npnt1 = 0, npnt2 = 0, nrade = 0, nrado = 0, npot = 0, ipot = 0, mblock = 0, nblock = 0;
    int grid_recs = 0;  // records before the level / block records of a file: 5, or 6 with r2
    bool zembed = false, zbisc = false;
    std::vector<int> nbass[2];
    std::vector<double> r1, r2, xd, wtd, dipol;
    DipoleFn fn{};
    double flops = 0.0;
    double dev_ms = 0.0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    ~Dip() {
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
    }
    // device work between begin() and end() is timed with events on the context's stream
    void begin() {
        if (!ev0) {
            CK(cudaEventCreate(&ev0));
            CK(cudaEventCreate(&ev1));
        }
        CK(cudaEventRecord(ev0, st));
    }
    void end() {
        CK(cudaEventRecord(ev1, st));
        CK(cudaEventSynchronize(ev1));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, ev0, ev1));
        dev_ms += ms;
    }

    // lagpt: points, weights and the weighted dipole at (r1(i1), r2(i2), xd(j)) in the order
    // trans reads it (i2 outer; symmetric Radau: i1 <= i2 - (1 - |nu|)).
    void lagpt(int nu) {
        std::vector<double> xh, wh;
        double csa, tsa;
        legendre_half(npot, xh, wh, csa, tsa);
        if (std::fabs((csa - tsa) / tsa) > 1.0e-8) bad(DVR3D_ERR_QUADRATURE, "DIPOLE3: gauss-legendre weights in error");
        const int n2 = npot / 2;
        xd.assign(npot, 0.0);
        wtd.assign(npot, 0.0);
        for (int i = 1; i <= n2; ++i) {
            xd[i - 1] = xh[i];
            wtd[i - 1] = wh[i];
        }
        for (int i = 1; i <= n2; ++i) {
            const int j = idia >= 0 ? i + n2 : npot + 1 - i;
            const int src = idia >= 0 ? npot - j + 1 : i;
            xd[j - 1] = -xd[src - 1];
            wtd[j - 1] = wtd[src - 1];
        }
        dipol.clear();
        const double scale = std::max(1, idia) == 2 ? 2.0 : 1.0;
        for (int i2 = 1; i2 <= npnt2; ++i2) {
            const double rr2 = idia == -2 ? r1[i2 - 1] : r2[i2 - 1];
            const int i0 = idia == -2 ? i2 - (1 - std::abs(nu)) : npnt1;
            for (int i1 = 1; i1 <= i0; ++i1)
                for (int j = 0; j < ipot; ++j) dipol.push_back(wtd[j] * (scale * fn(r1[i1 - 1], rr2, xd[j], nu)));
        }
    }

    // The ne states of block k (1-based) of side s at the angular points, on the device:
    // rows p = i + ipot mn (point i, radial function mn), nrad radial functions (dsrd).
    int amplitudes(int s, int k, int ip, int kk, int nu, double *A) {
        Wave &w = *W[s];
        const int n = ne[s], nb = nbass[s][k - 1];
        int nang = nb / nrade;
        if (ip == 1 && zbisc) nang = nb / nrado;
        const int nrad = (std::abs(nu) == 1 && ip == 0) ? nrade : nrado;
        const bool drop = nu == 0 && idia == -2 && ip == 0;  // the symmetric radial points go
        const int jdia = std::max(1, idia);
        int kz = kk;
        std::vector<double> fbr;  // (nang x nrad) per state, host, for files of J > 0
        std::vector<double> pk;   // (nang x nkept) for J = 0 files
        int iang = 0, nkept = 0;
        std::vector<double> v;    // packed vectors
        const std::string tg = std::to_string(s);
        if (nang < 1 || nrad < 1) bad(DVR3D_ERR_ARG, "DIPOLE3: block " + std::to_string(k) + " has no basis functions");
        if (jk[s] > 1) {
            // one record per k block: (ibase - 1) skipped states, then ne states of nbass each
            const size_t idx = (size_t)grid_recs + 1 + k;
            const double *rec = w.f.vec(idx, (size_t)nb * (ibase[s] - 1 + n)) + (size_t)nb * (ibase[s] - 1);
            if ((size_t)nang * (drop ? nrade : nrad) > (size_t)nb)
                bad(DVR3D_ERR_ARG, "DIPOLE3: radial parity of block " + std::to_string(k) + " does not match its size");
            v.resize((size_t)nang * nrad * n);
            for (int l = 0; l < n; ++l) {
                const double *src = rec + (size_t)l * nb;
                double *dst = &v[(size_t)l * nang * nrad];
                if (drop) {
                    int o = 0, q = 0;
                    for (int a = 1; a <= npnt1; ++a) {
                        for (int b = 1; b < a; ++b, ++o, ++q) std::memcpy(dst + (size_t)o * nang, src + (size_t)q * nang, 8 * (size_t)nang);
                        ++q;
                    }
                } else {
                    std::memcpy(dst, src, 8 * (size_t)nang * nrad);
                }
            }
        } else {
            // a J = 0 first-step file: the block's angular records, then its levels and states
            const size_t b0 = (size_t)grid_recs;
            auto kh = w.f.at(b0 + 1);
            if (kh.second < 12) bad(DVR3D_ERR_ARG, "wavefunction file: short k block header");
            int hk[3];
            std::memcpy(hk, kh.first, 12);
            kz = hk[0];
            const int maxleg = hk[1], nidvr = hk[2];
            const double *pl = w.f.vec(b0 + 2, (size_t)(maxleg + 1) * nidvr);
            std::vector<int> iv(nidvr, 1);
            int ibass = mbass[s];
            size_t vec0 = b0 + 5;
            iang = nidvr;
            if (zbisc) {
                auto ib = w.f.at(b0 + 3);
                auto ivr = w.f.at(b0 + 4);
                if (ib.second < 8 || ivr.second < 4 * (size_t)nidvr) bad(DVR3D_ERR_ARG, "wavefunction file: short selection records");
                int t2[2];
                std::memcpy(t2, ib.first, 8);
                iang = t2[0];
                ibass = t2[1];
                std::memcpy(iv.data(), ivr.first, 4 * (size_t)nidvr);
                vec0 = b0 + 7;
            }
            // jtran: the first angular function and the number of them
            int jstart = kz, jj0 = -jdia;
            const int par = zembed ? ipar[0] : ipar[s];
            if (idia == 2 && jstart % 2 != par) {
                ++jj0;
                ++jstart;
            }
            const int nt = (maxleg + kz - jstart) / jdia + 1;
            if (nt != nang) bad(DVR3D_ERR_ARG, "DIPOLE3: angular basis of the J = 0 file does not match its size");
            if (iang <= 0 || ibass < iang * (drop ? nrade : nrad))
                bad(DVR3D_ERR_ARG, "DIPOLE3: radial parity of the J = 0 file does not match its size");
            for (int a = 0; a < nidvr; ++a) nkept += iv[a] > 0;
            if (nkept > iang) bad(DVR3D_ERR_ARG, "wavefunction file: more kept angles than iang");
            pk.assign((size_t)nang * std::max(nkept, 1), 0.0);
            for (int a = 0, c = 0; a < nidvr; ++a) {
                if (iv[a] <= 0) continue;
                for (int j = 1; j <= nang; ++j) {
                    const int jj = jj0 + j * jdia;
                    if (jj > maxleg) bad(DVR3D_ERR_ARG, "DIPOLE3: angular function beyond the file's transform");
                    pk[(size_t)c * nang + (j - 1)] = pl[(size_t)a * (maxleg + 1) + jj];
                }
                ++c;
            }
            v.resize((size_t)iang * nrad * n);
            for (int l = 0; l < n; ++l) {
                const double *src = w.f.vec(vec0 + (size_t)(ibase[s] - 1) + l, (size_t)ibass);
                double *dst = &v[(size_t)l * iang * nrad];
                if (drop) {
                    int o = 0, q = 0;
                    for (int a = 1; a <= npnt1; ++a) {
                        for (int b = 1; b < a; ++b, ++o, ++q) std::memcpy(dst + (size_t)o * iang, src + (size_t)q * iang, 8 * (size_t)iang);
                        ++q;
                    }
                } else {
                    std::memcpy(dst, src, 8 * (size_t)iang * nrad);
                }
            }
        }
        // Legendre functions at the points (for Jacobi homonuclear files every other one)
        const std::vector<double> P = legendre_at(xd.size() == (size_t)ipot ? xd : std::vector<double>(xd.begin(), xd.begin() + ipot),
                                                  nang * jdia - 1, kz);
        std::vector<double> pd((size_t)ipot * nang);
        const int jfirst = idia == 2 ? (zembed ? (kk + ipar[0]) % 2 : (kk + ipar[s]) % 2) : 0;
        const int step = idia == 2 ? 2 : 1;
        for (int l = 0; l < nang; ++l)
            for (int i = 0; i < ipot; ++i) pd[(size_t)l * ipot + i] = P[(size_t)(jfirst + step * l) * ipot + i];
        double *dv = ctx->arena.get_t<double>("dp_v" + tg, v.size());
        double *dpd = ctx->arena.get_t<double>("dp_pd" + tg, pd.size());
        begin();
        CK(cudaMemcpyAsync(dv, v.data(), 8 * v.size(), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(dpd, pd.data(), 8 * pd.size(), cudaMemcpyHostToDevice, st));
        const double *fb = dv;
        if (jk[s] <= 1) {
            // angular DVR -> associated Legendre functions: FBR (nang x nrad n) = P'' V
            double *dpk = ctx->arena.get_t<double>("dp_pk" + tg, pk.size());
            double *df = ctx->arena.get_t<double>("dp_f" + tg, (size_t)nang * nrad * n);
            CK(cudaMemcpyAsync(dpk, pk.data(), 8 * pk.size(), cudaMemcpyHostToDevice, st));
            if (nkept > 0) {
                launch_dgemm(false, false, nang, nrad * n, nkept, 1.0, dpk, nang, dv, iang, 0.0, df, nang, st);
                CK(cudaGetLastError());
                flops += 2.0 * nang * nkept * (double)nrad * n;
            } else {
                CK(cudaMemsetAsync(df, 0, 8 * (size_t)nang * nrad * n, st));
            }
            fb = df;
        }
        // A (ipot x nrad n) = Pd (ipot x nang) FBR (nang x nrad n)
        launch_dgemm(false, false, ipot, nrad * n, nang, 1.0, dpd, ipot, fb, nang, 0.0, A, ipot, st);
        CK(cudaGetLastError());
        flops += 2.0 * ipot * nang * (double)nrad * n;
        end();  // also the host buffers v, pd, pk may go out of scope now
        return nrad;
    }

    // trans: T (ne0 x ne1) += A0^T diag(x1 w dipol) A1 over the points of this block
    void trans(double *T, const double *A0, int nrad0, const double *A1, int nrad1, int k1, int k2, double xfac,
               int nu, int ip) {
        const int j1 = jk[0] - kmin[0], j2 = jk[1] - kmin[1], kk1 = k1 - kmin[0], kk2 = k2 - kmin[1];
        double x1 = wigner3j(j1, 1, j2, kk1, nu, -kk2) * xfac;
        if (kk1 % 2 != 0) x1 = -x1;
        const int i0 = (std::abs(nu) == 1 && ip == 0) ? 0 : 1;
        std::vector<double> wv;
        size_t id = 0;
        for (int a = 1; a <= npnt1; ++a) {
            const int n0 = idia == -2 ? a - i0 : npnt2;
            const size_t cnt = (size_t)n0 * ipot;
            if (id + cnt > dipol.size()) bad(DVR3D_ERR_ARG, "DIPOLE3: dipole grid shorter than the block's points");
            for (size_t q = 0; q < cnt; ++q) wv.push_back(x1 * dipol[id + q]);
            id += cnt;
            if (std::abs(nu) == i0 && idia == -2) id += npot;
        }
        const int K = (int)wv.size();
        if (K > nrad0 * ipot || K > nrad1 * ipot) bad(DVR3D_ERR_ARG, "DIPOLE3: block vectors shorter than the points");
        if (K == 0) return;
        double *dw = ctx->arena.get_t<double>("dp_w", (size_t)K);
        double *S = ctx->arena.get_t<double>("dp_s", (size_t)K * ne[1]);
        begin();
        CK(cudaMemcpyAsync(dw, wv.data(), 8 * (size_t)K, cudaMemcpyHostToDevice, st));
        DVR3D_COUNT_LAUNCH(1);
        scale_rows_kernel<<<grid_for((long long)K * ne[1]), 256, 0, st>>>(A1, (long long)nrad1 * ipot, dw, K, ne[1], S);
        CK(cudaGetLastError());
        launch_dgemm(true, false, ne[0], ne[1], K, 1.0, A0, (long long)nrad0 * ipot, S, K, 1.0, T, ne[0], st);
        CK(cudaGetLastError());
        flops += 2.0 * ne[0] * ne[1] * (double)K;
        end();
    }
};

}  // namespace

void dipole3_run(dvr3d_ctx *ctx, const char *deck_text, const char *ket_path, const char *bra_path,
                 dvr3d_dipd_fn dipd, dvr3d_dipsa_fn dipsa, void *user, const char *tra_path,
                 dvr3d_dipole_result &res, std::string &text) {
    Dip D;
    D.ctx = ctx;
    D.st = ctx->stream;
    D.cd = read_cards(deck_text);
    if (D.cd.ires != 0) bad(DVR3D_ERR_UNSUPPORTED, "DIPOLE3 restart runs (IRES) are not built");
    Wave ket(ket_path), bra(bra_path);
    D.W[0] = &ket;
    D.W[1] = &bra;
    // ---- insize: consistency of the two files and the selection rules
    if (ket.idia != bra.idia) bad(DVR3D_ERR_ARG, "DIPOLE3: diatomic mismatch (idia)");
    D.idia = ket.idia;
    for (int s = 0; s < 2; ++s) {
        D.ipar[s] = D.W[s]->ipar;
        D.jrot[s] = D.W[s]->jrot;
        D.kmin[s] = D.W[s]->kmin;
    }
    if (D.jrot[0] == 0 && D.jrot[1] == 0) bad(DVR3D_ERR_ARG, "DIPOLE3: j = 0 -> 0 not allowed");
    if (D.jrot[0] == 0 || D.jrot[1] == 0) {
        D.zembed = D.jrot[0] == 0 ? bra.zemb : ket.zemb;
    } else if (D.idia > -2) {
        if (ket.zemb != bra.zemb) bad(DVR3D_ERR_ARG, "DIPOLE3: embedding mismatch");
        D.zembed = ket.zemb;
    }
    if (D.idia > -2) {
        if (D.idia == 2 && (D.zembed ? D.ipar[0] != D.ipar[1] : D.ipar[0] == D.ipar[1]))
            bad(DVR3D_ERR_ARG, "DIPOLE3: parity mismatch, spin forbidden");
        D.zbisc = false;
    } else {
        D.zbisc = true;
        D.zembed = true;
        if ((D.jrot[0] == D.jrot[1]) != (D.ipar[0] == D.ipar[1])) bad(DVR3D_ERR_ARG, "DIPOLE3: parity mismatch, spin forbidden");
    }
    if (ket.zmor1 != bra.zmor1 || ket.zmor2 != bra.zmor2) bad(DVR3D_ERR_ARG, "DIPOLE3: radial function mismatch");
    if (ket.nmax1 != bra.nmax1 || ket.nmax2 != bra.nmax2) bad(DVR3D_ERR_ARG, "DIPOLE3: radial DVR points differ");
    D.npnt1 = ket.nmax1;
    D.npnt2 = ket.nmax2;
    const double toler = 1.0e-3;
    if (std::fabs(bra.g1 - ket.g1) > toler || std::fabs(bra.g2 - ket.g2) > toler)
        bad(DVR3D_ERR_ARG, "DIPOLE3: co-ordinate system incompatible");
    for (int i = 0; i < 3; ++i)
        if (std::fabs(bra.xm[i] - ket.xm[i]) > toler) bad(DVR3D_ERR_ARG, "DIPOLE3: masses incompatible");
    for (int i = 0; i < 6; ++i)
        if (std::fabs(bra.morse[i] - ket.morse[i]) > toler) bad(DVR3D_ERR_ARG, "DIPOLE3: Morse parameters incompatible");
    if (ket.znco && bra.znco)
        bad(DVR3D_ERR_UNSUPPORTED, "DIPOLE3: both files without Coriolis coupling (ZNCOR) is not built");
    for (int s = 0; s < 2; ++s) {
        const Wave &w = *D.W[s];
        const Wave &o = *D.W[1 - s];
        if (w.znco && !o.znco) {
            if (std::abs(w.jrot) > 1) bad(DVR3D_ERR_ARG, "DIPOLE3: attempt to mix no coriolis and coupled calcs");
            D.kmin[s] = 0;
        }
    }
    for (int s = 0; s < 2; ++s) {
        if (D.jrot[s] == 0) D.kmin[s] = 1;
        D.jk[s] = D.jrot[s] + D.kmin[s];
    }
    D.mblock = D.jk[0] + D.jk[1] + std::min(D.jk[0], D.jk[1]) - 2;
    D.nblock = std::min(D.cd.nblock, D.mblock);
    if (D.idia > -2) {
        D.nrade = D.nrado = D.npnt1 * D.npnt2;
        for (int s = 0; s < 2; ++s) D.mbass[s] = D.nrade * D.jk[s] * D.W[s]->lmax;
    } else {
        D.nrade = D.npnt1 * (D.npnt1 + 1) / 2;
        D.nrado = D.npnt1 * (D.npnt1 - 1) / 2;
        for (int s = 0; s < 2; ++s) {
            const int jt = D.jk[s] / 2;
            int m = (D.nrade + D.nrado) * jt;
            if (2 * jt != D.jk[s]) m += D.ipar[s] == 0 ? D.nrade : D.nrado;
            D.mbass[s] = m * D.W[s]->lmax;
        }
    }
    const int nv[2] = {D.cd.nv1, D.cd.nv2};
    D.ibase[0] = D.cd.ibase1;
    D.ibase[1] = D.cd.ibase2;
    for (int s = 0; s < 2; ++s) {
        const int nev = D.W[s]->neval;
        if (D.ibase[s] <= 0 || D.ibase[s] > nev) D.ibase[s] = 1;
        D.ne[s] = nv[s] > 0 ? std::min(nv[s], nev - D.ibase[s] + 1) : nev - D.ibase[s] + 1;
        if (D.ne[s] < 1) bad(DVR3D_ERR_ARG, "DIPOLE3: no states to take from a file");
    }
    const int itot = D.jrot[0] + D.jrot[1] + 1 + D.kmin[0] + D.kmin[1];
    if (itot % 2 != 0 || std::abs(D.jrot[0] - D.jrot[1]) > 1) bad(DVR3D_ERR_ARG, "DIPOLE3: selection rules violated");
    D.npot = D.cd.npot + (D.cd.npot % 2);
    if (D.npot < 2) bad(DVR3D_ERR_DECK, "DIPOLE3: NPOT must be at least 2");
    D.ipot = D.idia < 2 ? D.npot : D.npot / 2;
    D.fn = DipoleFn{dipd, dipsa, user, ket.g1, bra.g2, D.zembed, D.zbisc};
    // ---- genind: (mbass0, lmin, lbass, nbass) of each file
    for (int s = 0; s < 2; ++s) {
        auto r = D.W[s]->f.at(3);
        const int jk = D.jk[s];
        if (r.second < 4 * (size_t)(1 + 3 * jk)) bad(DVR3D_ERR_ARG, "wavefunction file: basis function labels too short");
        std::vector<int> a(1 + 3 * jk);
        std::memcpy(a.data(), r.first, 4 * a.size());
        if (a[0] > D.mbass[s]) bad(DVR3D_ERR_ARG, "DIPOLE3: basis function dimensions in error");
        D.nbass[s].assign(a.begin() + 1 + 2 * jk, a.end());
    }
    // ---- radial grid (from the bra), levels
    D.grid_recs = D.idia > -2 ? 6 : 5;
    {
        const double *g = bra.f.vec(4, (size_t)D.npnt1);
        D.r1.assign(g, g + D.npnt1);
        if (D.idia > -2) {
            const double *g2 = bra.f.vec(5, (size_t)D.npnt2);
            D.r2.assign(g2, g2 + D.npnt2);
        }
    }
    std::vector<double> e[2];
    for (int s = 0; s < 2; ++s) {
        const size_t lev = (size_t)D.grid_recs + (D.jk[s] <= 1 ? (D.idia == -2 ? 5 : 3) : 0);
        const double *ev = D.W[s]->f.vec(lev + 1, (size_t)(D.ibase[s] - 1 + D.ne[s]));
        e[s].assign(ev + D.ibase[s] - 1, ev + D.ibase[s] - 1 + D.ne[s]);
    }
    if (res.cap1 < D.ne[0] || res.cap2 < D.ne[1]) bad(DVR3D_ERR_BUFFER, "DIPOLE3: result buffers smaller than the states taken");
    // ---- dmain: the k -> k' blocks
    cudaStream_t st = D.st;
    const int n0 = D.ne[0], n1 = D.ne[1];
    double *Tz = ctx->arena.get_t<double>("dp_tz", (size_t)n0 * n1);
    double *Tx = ctx->arena.get_t<double>("dp_tx", (size_t)n0 * n1);
    CK(cudaMemsetAsync(Tz, 0, 8 * (size_t)n0 * n1, st));
    CK(cudaMemsetAsync(Tx, 0, 8 * (size_t)n0 * n1, st));
    auto amp_buf = [&](const std::string &name, int nrad_max, int s) {
        return ctx->arena.get_t<double>(name, (size_t)nrad_max * D.ipot * D.ne[s]);
    };
    const int nrmax = std::max(D.nrade, D.nrado);
    std::string log;
    char ln[256];
    int iblock = 0;
    bool stop = false;
    int ipar11 = D.ipar[0], ipar22 = D.ipar[1];  // the phase convention of symmetric Radau
    if (D.idia == -2) {
        if (D.kmin[0] == 0) ipar11 += 1;
        if (D.kmin[1] == 0) ipar22 += 1;
    }
    auto phase = [&](int kk1, int kk2) { return D.idia == -2 && ((kk1 + ipar11) / 2 + (kk2 + ipar22) / 2) % 2 != 0; };
    auto note = [&](int k1, int k2, bool done) {
        std::snprintf(ln, sizeof(ln), "\n     Block%4d k1 =%3d to k2 =%3d %s\n", iblock, k1 - D.kmin[0], k2 - D.kmin[1],
                      done ? "completed" : "skipped");
        log += ln;
    };
    // nu = 0: k1 -> k2 = k1 - kmin1 + kmin2
    D.lagpt(0);
    {
        int ks1 = 1, ip = D.ipar[0];
        if (D.kmin[0] > D.kmin[1]) {
            ks1 = 2;
            ip = 1 - ip;
        }
        double *A0 = amp_buf("dp_a0", nrmax, 0), *A1 = amp_buf("dp_a1", nrmax, 1);
        for (int k1 = ks1; k1 <= D.jk[0] && !stop; ++k1, ip = 1 - ip) {
            const int k2 = k1 - D.kmin[0] + D.kmin[1];
            if (k2 > D.jk[1]) continue;
            ++iblock;
            if (D.nbass[0][k1 - 1] == 0 || D.nbass[1][k2 - 1] == 0) {
                note(k1, k2, false);
                continue;
            }
            const int kk = k1 - D.kmin[0];
            const int na = D.amplitudes(0, k1, ip, kk, 0, A0);
            const int nb = D.amplitudes(1, k2, 1 - ip, kk, 0, A1);
            D.trans(Tz, A0, na, A1, nb, k1, k2, phase(kk, kk) ? -1.0 : 1.0, 0, 1);
            note(k1, k2, true);
            if (iblock >= D.nblock) stop = true;
        }
    }
    // nu = +1, -1: k1 -> k2 with kk2 = kk1 +/- 1; each bra block evaluated once, with the
    // radial parity ip of the ket blocks that use it
    if (!stop) {
        D.lagpt(1);
        double *A0 = amp_buf("dp_a0", nrmax, 0);
        double *slot[3] = {amp_buf("dp_b0", nrmax, 1), amp_buf("dp_b1", nrmax, 1), amp_buf("dp_b2", nrmax, 1)};
        int held[3] = {-1, -1, -1}, hnrad[3] = {0, 0, 0}, hip[3] = {-1, -1, -1};
        auto bra_amp = [&](int k2, int ip, int &nrad) -> const double * {
            const int q = k2 % 3;
            if (held[q] != k2 || hip[q] != ip) {
                hnrad[q] = D.amplitudes(1, k2, ip, k2 - D.kmin[1], 1, slot[q]);
                held[q] = k2;
                hip[q] = ip;
            }
            nrad = hnrad[q];
            return slot[q];
        };
        int ip = D.ipar[0];
        for (int k1 = 1; k1 <= D.jk[0] && !stop; ++k1, ip = 1 - ip) {
            const int kk1 = k1 - D.kmin[0];
            if (D.nbass[0][k1 - 1] == 0) continue;
            const int na = D.amplitudes(0, k1, ip, kk1, 1, A0);
            for (int nu : {1, -1}) {
                if (nu == 1 && D.jk[1] <= 1) continue;
                const int kk2 = kk1 + nu, k2 = kk2 + D.kmin[1];
                if (k2 < 1 || k2 > D.jk[1]) continue;
                ++iblock;
                if (D.nbass[1][k2 - 1] == 0) {
                    note(k1, k2, false);
                    continue;
                }
                double xfac;
                if (nu == 1) xfac = kk1 == 0 ? -1.0 : -1.0 / std::sqrt(2.0);
                else xfac = kk2 == 0 ? 1.0 : 1.0 / std::sqrt(2.0);
                if (phase(kk1, kk2)) xfac = -xfac;
                if (!D.zembed && D.idia < 0) xfac = -xfac;
                int nb = 0;
                const double *B = bra_amp(k2, ip, nb);
                D.trans(Tx, A0, na, B, nb, k1, k2, xfac, nu, ip);
                note(k1, k2, true);
                if (iblock >= D.nblock && (nu == 1 || k1 < D.jk[0])) {
                    stop = true;
                    break;
                }
            }
        }
    }
    std::vector<double> tz((size_t)n0 * n1), tx((size_t)n0 * n1);
    CK(cudaMemcpyAsync(tz.data(), Tz, 8 * tz.size(), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(tx.data(), Tx, 8 * tx.size(), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    // ---- spect: line strengths, Einstein coefficients, the printed table
    const double autocm = 2.19474624e+05, autode = 2.5417662, detosec = 3.136186e-07;
    const int j1 = D.jk[0] - D.kmin[0], j2 = D.jk[1] - D.kmin[1];
    const double ez = D.cd.ezero;
    std::string s = log;
    std::snprintf(ln, sizeof(ln), "\n     %s\n", D.cd.title.c_str());
    s += ln;
    std::snprintf(ln, sizeof(ln), "\n     j1=%4d  kmin1=%4d  j2=%4d  kmin2=%4d  idia=%4d  ipar1=%4d  ipar2=%4d\n\n", j1,
                  D.kmin[0], j2, D.kmin[1], D.idia, D.ipar[0], D.ipar[1]);
    s += ln;
    if (D.cd.have_ezero) s += "     ground zero =" + fortran_e(ez, 16, 8, 'E') + " cm-1\n";
    s += "\n ie1 ie2   ket energy   bra energy    frequency  z transition    x transition       dipole       s(f-i)"
         "      a-coefficient\n\n";
    const double xf = std::sqrt((double)((2 * j1 + 1) * (2 * j2 + 1)));
    std::vector<double> sint((size_t)n0 * n1);
    for (int a = 0; a < n0; ++a) {
        const double xe1 = e[0][a] * autocm - ez;
        for (int b = 0; b < n1; ++b) {
            const double xe2 = e[1][b] * autocm - ez;
            const double dd = xe2 - xe1, dd3 = std::fabs(dd * dd * dd);
            const size_t q = (size_t)a + (size_t)n0 * b;
            const double sum = tz[q] + tx[q];
            sint[q] = sum * sum * xf * xf;
            const double tzd = tz[q] * autode * xf;
            const double txd = (!D.zbisc && D.zembed) ? -tx[q] * autode * xf : tx[q] * autode * xf;
            const double t = std::fabs(tzd + txd), sxd = t * t;
            const double acoef = dd > 0.0 ? sxd * dd3 * detosec / (2 * j2 + 1) : (dd < 0.0 ? sxd * dd3 * detosec / (2 * j1 + 1) : 0.0);
            if (D.cd.zpmin && std::max(a, b) + 1 > 10) continue;
            std::snprintf(ln, sizeof(ln), "%4d%4d   %14.6f   %14.6f   %14.6f  %s  %s  %s  %s  %s\n", a + 1, b + 1, xe1, xe2,
                          dd, fortran_es(tzd, 15, 8).c_str(), fortran_es(txd, 15, 8).c_str(),
                          fortran_es(t, 15, 8).c_str(), fortran_es(sxd, 15, 8).c_str(), fortran_es(acoef, 15, 8).c_str());
            s += ln;
        }
    }
    text = s;
    // ---- outpt: the records for program SPECTRA
    if (D.cd.ztra && tra_path && tra_path[0]) {
        FILE *fp = std::fopen(tra_path, D.cd.zstart ? "wb" : "ab");
        if (!fp) bad(DVR3D_ERR_ARG, std::string("cannot open ") + tra_path);
        struct Closer {
            FILE *f;
            ~Closer() { std::fclose(f); }
        } closer{fp};
        RecordWriter w{fp};
        for (int v : {j1, j2, D.kmin[0], D.kmin[1], n0, n1, D.idia, D.ipar[0], D.ipar[1]}) w.i4(v);
        w.r8(ez);
        w.i4(D.zembed ? 1 : 0);
        w.i4(D.ibase[0]);
        w.i4(D.ibase[1]);
        w.end();
        for (double v : e[0]) w.r8(v);
        w.end();
        for (double v : e[1]) w.r8(v);
        w.end();
        for (int b = 0; b < n1; ++b) {
            w.put(&sint[(size_t)n0 * b], 8 * (size_t)n0);
            w.end();
        }
    }
    // ---- results
    res.neval1 = n0;
    res.neval2 = n1;
    res.j1 = j1;
    res.j2 = j2;
    res.kmin1 = D.kmin[0];
    res.kmin2 = D.kmin[1];
    res.nblocks = iblock;
    res.dev_ms = D.dev_ms;
    res.flops = D.flops;
    auto put = [&](double *dst, const std::vector<double> &src) {
        if (!dst) return;
        for (int b = 0; b < n1; ++b)
            std::memcpy(dst + (size_t)res.cap1 * b, &src[(size_t)n0 * b], 8 * (size_t)n0);
    };
    put(res.tz, tz);
    put(res.tx, tx);
    put(res.sint, sint);
    if (res.e1) std::memcpy(res.e1, e[0].data(), 8 * (size_t)n0);
    if (res.e2) std::memcpy(res.e2, e[1].data(), 8 * (size_t)n1);
}

}  // namespace dvr3d
