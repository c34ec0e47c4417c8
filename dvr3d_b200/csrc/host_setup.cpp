// host_setup.cpp -- job-deck reading and the FP64 set-up of one k block.
//
// The quadrature routines reproduce the reference's iteration steps exactly (start values,
// search steps, Newton stopping rules and the point at which derivatives are taken): the
// reference's Gauss weights carry iteration-history errors of ~1e-11 relative (its printed
// "computed sum of weights" is 1.99999999999202 for NALF=40) and those errors reach the
// final levels at the 1e-6 cm-1 level, so a different root finder would not be a drop-in.
#include "host_setup.h"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <sstream>

namespace dvr3d {

namespace {

[[noreturn]] void raise(int code, const std::string &msg) { throw HostError{code, msg}; }

// ------------------------------------------------------------------ deck reading
std::string upper(std::string s) {
    for (auto &c : s) c = (char)std::toupper((unsigned char)c);
    return s;
}

// Fortran formatted integer field (Iw, BLANK='NULL': blanks ignored, empty field = 0).
int int_field(const std::string &line, size_t col, size_t width) {
    std::string f;
    for (size_t i = col; i < col + width && i < line.size(); ++i)
        if (line[i] != ' ' && line[i] != '\t' && line[i] != '\r') f += line[i];
    if (f.empty()) return 0;
    char *end = nullptr;
    long v = std::strtol(f.c_str(), &end, 10);
    if (*end != '\0') raise(DVR3D_ERR_DECK, "bad integer field '" + f + "'");
    return (int)v;
}

// Fortran formatted real field (Fw.0): blanks ignored, D exponents accepted, a field
// without a decimal point is an integer value (scale 0).
double real_field(const std::string &line, size_t col, size_t width) {
    std::string f;
    for (size_t i = col; i < col + width && i < line.size(); ++i) {
        char c = line[i];
        if (c == ' ' || c == '\t' || c == '\r') continue;
        if (c == 'd' || c == 'D' || c == 'q' || c == 'Q') c = 'E';
        f += c;
    }
    if (f.empty()) return 0.0;
    char *end = nullptr;
    double v = std::strtod(f.c_str(), &end);
    if (*end != '\0') raise(DVR3D_ERR_DECK, "bad real field '" + f + "'");
    return v;
}

void set_defaults(dvr3d_deck &d) {
    std::memset(&d, 0, sizeof(d));
    // block data :158-167
    d.zpham = 0; d.zprad = 0; d.zpvec = 0; d.zrot = 1; d.zladd = 1; d.zembed = 1;
    d.zmors2 = 1; d.zpmin = 0; d.zvec = 0; d.zquad2 = 1; d.zcut = 0; d.zdiag = 1;
    d.zlmat = 0; d.zall = 0; d.zp1d = 0; d.zp2d = 0; d.zr2r1 = 1; d.ztheta = 1;
    d.zmors1 = 1; d.ztran = 0; d.ztwod = 0; d.zperp = 0; d.zx = 0; d.zs0 = 0; d.zs1 = 0;
    d.zlin = 0; d.zpfun = 0;
    d.ncoord = 3;
}

int *logical_slot(dvr3d_deck &d, const std::string &name) {
    struct E { const char *n; int dvr3d_deck::*m; };
    static const E tab[] = {
        {"ZPHAM", &dvr3d_deck::zpham}, {"ZPRAD", &dvr3d_deck::zprad},
        {"ZPVEC", &dvr3d_deck::zpvec}, {"ZROT", &dvr3d_deck::zrot},
        {"ZLADD", &dvr3d_deck::zladd}, {"ZEMBED", &dvr3d_deck::zembed},
        {"ZMORS2", &dvr3d_deck::zmors2}, {"ZS0", &dvr3d_deck::zs0},
        {"ZX", &dvr3d_deck::zx}, {"ZS1", &dvr3d_deck::zs1}, {"ZPMIN", &dvr3d_deck::zpmin},
        {"ZVEC", &dvr3d_deck::zvec}, {"ZQUAD2", &dvr3d_deck::zquad2},
        {"ZDIAG", &dvr3d_deck::zdiag}, {"ZLMAT", &dvr3d_deck::zlmat},
        {"ZCUT", &dvr3d_deck::zcut}, {"ZALL", &dvr3d_deck::zall}, {"ZLIN", &dvr3d_deck::zlin},
        {"ZP1D", &dvr3d_deck::zp1d}, {"ZP2D", &dvr3d_deck::zp2d},
        {"ZR2R1", &dvr3d_deck::zr2r1}, {"ZTHETA", &dvr3d_deck::ztheta},
        {"ZTRAN", &dvr3d_deck::ztran}, {"ZMORS1", &dvr3d_deck::zmors1},
        {"ZTWOD", &dvr3d_deck::ztwod}, {"ZPERP", &dvr3d_deck::zperp},
        {"ZPFUN", &dvr3d_deck::zpfun}};
    for (const auto &e : tab)
        if (name == e.n) return &(d.*(e.m));
    return nullptr;
}

bool is_unit_name(const std::string &n) {
    static const char *units[] = {"IDIAG1", "IDIAG2", "IOUT1", "IOUT2", "IWAVE", "ILEV",
                                  "IEIGS1", "IVECS1", "IEIGS2", "IVECS2", "IVINT", "IBAND",
                                  "INTVEC"};
    for (auto u : units)
        if (n == u) return true;
    return false;
}

// Namelist /PRT/ (dvr3d :54-58,:65). Returns the index of the first line after it.
size_t read_namelist(const std::vector<std::string> &lines, dvr3d_deck &d) {
    size_t li = 0;
    while (li < lines.size() && lines[li].find_first_not_of(" \t\r") == std::string::npos) ++li;
    if (li >= lines.size()) raise(DVR3D_ERR_DECK, "empty deck");
    std::string first = upper(lines[li]);
    size_t amp = first.find('&');
    if (amp == std::string::npos) raise(DVR3D_ERR_DECK, "deck must start with namelist &PRT");
    size_t p = amp + 1;
    std::string grp;
    while (p < first.size() && std::isalnum((unsigned char)first[p])) grp += first[p++];
    if (grp != "PRT") raise(DVR3D_ERR_DECK, "namelist group must be PRT, got " + grp);
    // gather the text up to the terminating '/' (or &END)
    std::string body = first.substr(p);
    size_t end_line = li;
    auto terminated = [](const std::string &s, size_t &cut) {
        size_t sl = s.find('/');
        size_t en = s.find("&END");
        cut = std::min(sl, en);
        return cut != std::string::npos;
    };
    size_t cut;
    while (!terminated(body, cut)) {
        ++end_line;
        if (end_line >= lines.size()) raise(DVR3D_ERR_DECK, "namelist not terminated by /");
        body += " " + upper(lines[end_line]);
    }
    body = body.substr(0, cut);
    for (auto &c : body)
        if (c == ',' || c == '\t' || c == '\r') c = ' ';
    // tokens name = value
    std::vector<std::string> tok;
    {
        std::string cur;
        for (char c : body) {
            if (c == '=') {
                if (!cur.empty()) tok.push_back(cur);
                tok.push_back("=");
                cur.clear();
            } else if (c == ' ') {
                if (!cur.empty()) tok.push_back(cur);
                cur.clear();
            } else {
                cur += c;
            }
        }
        if (!cur.empty()) tok.push_back(cur);
    }
    for (size_t i = 0; i < tok.size();) {
        if (i + 2 >= tok.size() + 0 && !(i + 2 < tok.size() + 1)) break;
        if (i + 2 > tok.size() || tok[i + 1] != "=")
            raise(DVR3D_ERR_DECK, "malformed namelist entry near '" + tok[i] + "'");
        if (i + 2 >= tok.size()) raise(DVR3D_ERR_DECK, "missing value for " + tok[i]);
        const std::string &name = tok[i], &val = tok[i + 2];
        if (int *slot = logical_slot(d, name)) {
            std::string v = val;
            if (!v.empty() && v[0] == '.') v = v.substr(1);
            if (v.empty() || (v[0] != 'T' && v[0] != 'F'))
                raise(DVR3D_ERR_DECK, "bad logical value for " + name);
            *slot = (v[0] == 'T') ? 1 : 0;
        } else if (is_unit_name(name)) {
            // unit numbers of scratch/output streams: accepted, not used by this library
        } else {
            raise(DVR3D_ERR_DECK, "unknown namelist variable " + name);
        }
        i += 3;
    }
    return end_line + 1;
}

}  // namespace

void parse_deck(const std::string &text, dvr3d_deck &d) {
    set_defaults(d);
    std::vector<std::string> lines;
    {
        std::string cur;
        for (char c : text) {
            if (c == '\n') {
                lines.push_back(cur);
                cur.clear();
            } else {
                cur += c;
            }
        }
        if (!cur.empty()) lines.push_back(cur);
    }
    size_t li = read_namelist(lines, d);
    auto line = [&](size_t i) -> std::string { return i < lines.size() ? lines[i] : std::string(); };
    auto need = [&](size_t i, const char *what) {
        if (i >= lines.size()) raise(DVR3D_ERR_DECK, std::string("deck ends before ") + what);
    };
    need(li, "card 2 (NCOORD)");
    d.ncoord = int_field(line(li), 0, 5);  // insize :232 format 15i5
    ++li;
    need(li, "card 3");
    {
        std::string c = line(li);
        int *f[11] = {&d.npnt2, &d.jrot, &d.neval, &d.nalf, &d.max2d, &d.max3d,
                      &d.idia, &d.kmin, &d.npnt1, &d.ipar, &d.max3d2};
        for (int k = 0; k < 11; ++k) *f[k] = int_field(c, 5 * k, 5);  // :238-239
    }
    ++li;
    {
        std::string t = line(li);  // title 9a8 (:372)
        if (t.size() > 72) t = t.substr(0, 72);
        std::strncpy(d.title, t.c_str(), sizeof(d.title) - 1);
    }
    ++li;
    // setcon cards (:1042-1095), format 3f20.0
    d.fixcos = real_field(line(li), 0, 20);
    ++li;
    need(li, "the XMASS card");
    for (int k = 0; k < 3; ++k) d.xmass[k] = real_field(line(li), 20 * k, 20);
    ++li;
    for (int k = 0; k < 3; ++k) d.xmassr[k] = real_field(line(li), 20 * k, 20);
    ++li;
    d.emax1 = real_field(line(li), 0, 20);
    d.emax2 = real_field(line(li), 20, 20);
    ++li;
    d.re1 = real_field(line(li), 0, 20);
    d.diss1 = real_field(line(li), 20, 20);
    d.we1 = real_field(line(li), 40, 20);
    ++li;
    d.re2 = real_field(line(li), 0, 20);
    d.diss2 = real_field(line(li), 20, 20);
    d.we2 = real_field(line(li), 40, 20);
    ++li;
    // optional EZERO card read by diag3d for odd parity (:2751, format f20.0)
    d.have_ezero = 0;
    if (li < lines.size() && lines[li].find_first_not_of(" \t\r") != std::string::npos) {
        d.ezero = real_field(lines[li], 0, 20);
        d.have_ezero = 1;
    }
}

namespace {

const double kAmToAu = 1.8228883e03;  // setcon :1037
const double kAuToCm = 2.19474624e+05;  // diag3d :2681

// Three-term recurrence value/derivative/previous value of the monic Laguerre-type
// polynomial p_n(x) of laguer/lgrecr (:1466-1492).
struct LagRec {
    int n;
    double alf;
    std::vector<double> b, c;  // 1-based as in the recurrence definition
    void eval(double x, double &pn, double &dpn, double &pn1) const {
        double p1 = 1.0, p = x - alf - 1.0, dp1 = 0.0, dp = 1.0;
        for (int j = 2; j <= n; ++j) {
            const double q = (x - b[j]) * p - c[j] * p1;
            const double dq = (x - b[j]) * dp - c[j] * dp1 + p;
            p1 = p;
            p = q;
            dp1 = dp;
            dp = dq;
        }
        pn = p;
        dpn = dp;
        pn1 = p1;
    }
};

// Gauss-Laguerre points and pseudo-weights for weight y^alf e^-y (laguer :1369-1436).
void gauss_laguerre(int n, double alf, double cc, std::vector<double> &x, std::vector<double> &w,
                    double &csx, double &csa, double &tsx) {
    LagRec R{n, alf, std::vector<double>(n + 2), std::vector<double>(n + 2)};
    double fa = alf + 1.0, fn = 1.0;
    R.b[1] = fa;
    R.c[1] = 0.0;
    for (int j = 2; j <= n; ++j) {
        fa += 2.0;
        R.b[j] = fa;
        R.c[j] = fn * (alf + fn);
        fn += 1.0;
    }
    tsx = fn * (alf + fn);
    x.assign(n, 0.0);
    w.assign(n, 0.0);
    csx = csa = 0.0;
    double prev1 = 0.0, prev2 = 0.0;  // last two roots (xt1, xt2 of the reference)
    double xt = (1.0 + alf) * (2.0 + alf) / (1.0 + 3.0 * fn + 2.0 * alf);
    const double step = 3.0 * (1.0 + alf) / (1.0 + 3.0 * fn + alf);
    double pt, dpn, pn1, pt2;
    R.eval(xt, pt, dpn, pn1);
    for (int i = 1; i <= n; ++i) {
        if (i <= 2) {
            // march right in fixed steps until p changes sign, start at the midpoint
            for (;;) {
                const double xs = xt + step;
                R.eval(xs, pt2, dpn, pn1);
                const bool same = (pt >= 0.0) == (pt2 >= 0.0);
                pt = pt2;
                if (same) {
                    xt = xs;
                    continue;
                }
                prev2 = xs;
                xt = 0.5 * (xt + xs);
                break;
            }
        } else {
            const double fi = (double)(i - 2);
            const double q1 = (1.0 + 2.55 * fi) / (1.9 * fi);
            const double q2 = 1.26 * fi * alf / (1.0 + 3.5 * fi);
            xt = xt + (q1 + q2) / (1.0 + 0.3 * alf) * (xt - prev2);
        }
        // Newton with relative stopping 1e-12, at most 10 steps (lgroot :1439-1463);
        // the derivative and p_{n-1} are those of the last evaluation before the update.
        for (int it = 1;; ++it) {
            double p;
            R.eval(xt, p, dpn, pn1);
            const double d = p / dpn;
            xt -= d;
            if (std::fabs(d / xt) <= 1.0e-12 || it >= 10) break;
        }
        prev2 = prev1;
        prev1 = xt;
        x[i - 1] = xt;
        w[i - 1] = cc / dpn / pn1;
        csx += xt;
        csa += w[i - 1];
    }
}

// ln Gamma(x) by the six-term Lanczos series the reference uses (gammln :4265-4286); its
// coefficients are kept so that the z-perp weights and polynomial norms match the
// reference's to the last digits it prints.
double lanczos_lngamma(double xx) {
    constexpr double c[6] = {76.18009173, -86.50532033, 24.01409822, -1.231739516, 0.120858003e-2, -0.536382e-5};
    double x = xx - 1.0;
    const double t = x + 5.5;
    const double lead = (x + 0.5) * std::log(t) - t;
    double ser = 1.0;
    for (double cj : c) {
        x += 1.0;
        ser += cj / x;
    }
    return lead + std::log(2.50662827465 * ser);
}

// n-point Gauss-Jacobi rule for the weight (1-x)^a (1+x)^b, points descending from +1
// (gaujac :4190-4263): Newton iteration on the three-term recurrence, stopping at 3e-14 or
// 10 steps, from the reference's asymptotic first guesses (one of its constants is a REAL*4
// literal, 0.012, and is used as such).
void gauss_jacobi_full(int n, double a, double b, std::vector<double> &x, std::vector<double> &w) {
    x.assign(n, 0.0);
    w.assign(n, 0.0);
    const double dn = n, nn = (double)(n * n), ab = a + b;
    double z = 0.0;
    for (int i = 0; i < n; ++i) {
        const int ii = i + 1;
        if (ii == 1) {
            const double an = a / dn, bn = b / dn;
            z = 1.0 - (1.0 + a) * (2.78 / (4.0 + nn) + 0.768 * an / dn) /
                          (1.0 + 1.48 * an + 0.96 * bn + 0.452 * an * an + 0.83 * an * bn);
        } else if (ii == 2) {
            z -= (1.0 - z) * ((4.1 + a) / ((1.0 + a) * (1.0 + 0.156 * a))) *
                 (1.0 + 0.06 * (dn - 8.0) * (1.0 + 0.12 * a) / dn) *
                 (1.0 + (double)0.012f * b * (1.0 + 0.25 * std::fabs(a)) / dn);
        } else if (ii == 3) {
            z -= (x[0] - z) * ((1.67 + 0.28 * a) / (1.0 + 0.37 * a)) * (1.0 + 0.22 * (dn - 8.0) / dn) *
                 (1.0 + 8.0 * b / ((6.28 + b) * nn));
        } else if (ii == n - 1) {
            z += (z - x[n - 4]) * ((1.0 + 0.235 * b) / (0.766 + 0.119 * b)) *
                 (1.0 / (1.0 + 0.639 * (dn - 4.0) / (1.0 + 0.71 * (dn - 4.0)))) *
                 (1.0 / (1.0 + 20.0 * a / ((7.5 + a) * nn)));
        } else if (ii == n) {
            z += (z - x[n - 3]) * ((1.0 + 0.37 * b) / (1.67 + 0.28 * b)) *
                 (1.0 / (1.0 + 0.22 * (double)(n - 8) / dn)) * (1.0 / (1.0 + 8.0 * a / ((6.28 + a) * nn)));
        } else {
            z = 3.0 * x[i - 1] - 3.0 * x[i - 2] + x[i - 3];
        }
        double p1 = 0.0, p2 = 0.0, dp = 0.0, t = 0.0;
        for (int it = 0; it < 10; ++it) {
            t = 2.0 + ab;
            p1 = (a - b + t * z) / 2.0;
            p2 = 1.0;
            for (int j = 2; j <= n; ++j) {
                const double p3 = p2;
                p2 = p1;
                t = 2.0 * j + ab;
                const double c1 = 2.0 * j * (j + ab) * (t - 2.0);
                const double c2 = (t - 1.0) * (a * a - b * b + t * (t - 2.0) * z);
                const double c3 = 2.0 * (j - 1 + a) * (j - 1 + b) * t;
                p1 = (c2 * p2 - c3 * p3) / c1;
            }
            dp = (dn * (a - b - t * z) * p1 + 2.0 * (dn + a) * (dn + b) * p2) / (t * (1.0 - z * z));
            const double zold = z;
            z = zold - p1 / dp;
            if (std::fabs(z - zold) <= 3.0e-14) break;
        }
        x[i] = z;
        w[i] = std::exp(lanczos_lngamma(a + dn) + lanczos_lngamma(b + dn) - lanczos_lngamma(dn + 1.0) -
                        lanczos_lngamma(dn + ab + 1.0)) *
               t * std::pow(2.0, ab) / (dp * p2);
    }
}

// Normalised Jacobi polynomials P_l^(a,b)(x_i), l = 0..lmax, at the points x (jac_basis
// :4136-4154, jacgt :4158-4186, norms2 :4288-4308); column i of the result holds point i.
std::vector<double> jacobi_poly_basis(const std::vector<double> &x, int npt, int lmax, double a, double b) {
    const double lam = a + b + 1.0;
    std::vector<double> out((size_t)(lmax + 1) * npt);
    std::vector<double> nrm(lmax + 1);
    for (int l = 0; l <= lmax; ++l)
        nrm[l] = std::sqrt(std::pow(2.0, -lam) * (2.0 * l + lam) *
                           std::exp(lanczos_lngamma(l + 1.0) + lanczos_lngamma(l + lam) - lanczos_lngamma(l + a + 1.0) -
                                    lanczos_lngamma(l + b + 1.0)));
    for (int i = 0; i < npt; ++i) {
        double *col = &out[(size_t)i * (lmax + 1)];
        col[0] = 1.0;
        if (lmax >= 1) col[1] = (a - b + (lam + 1.0) * x[i]) / 2.0;
        for (int l = 2; l <= lmax; ++l) {
            const int m = l - 1;  // recurrence coefficients of degree m
            const double d1 = 2.0 * (m + 1.0) * (m + lam) * (2.0 * m + lam - 1.0);
            const double d2 = (2.0 * m + lam) * (a * a - b * b);
            const double d3 = (2.0 * m + lam - 1.0) * (2.0 * m + lam) * (2.0 * m + lam + 1.0);
            const double d4 = 2.0 * (m + a) * (m + b) * (2.0 * m + lam + 1.0);
            col[l] = ((d2 + d3 * x[i]) * col[l - 1] - d4 * col[l - 2]) / d1;
        }
        for (int l = 0; l <= lmax; ++l) col[l] *= nrm[l];
    }
    return out;
}

// Gauss-Jacobi (alpha = beta = nu) roots on the half range and weights, found by the
// reference's downward sign scan from x=1 in REAL*4 steps of 1e-4 followed by Newton with
// absolute stopping 1e-12 (jacobi :1635-1699, root :1702-1721, recur :1722-1744).
void gauss_jacobi_half(int n, int n2, double nu, double tsa, std::vector<double> &x,
                       std::vector<double> &w, double &csa) {
    std::vector<double> c(n + 2, 0.0);
    for (int i = 2; i <= n; ++i) {
        const double xi = (double)i, s = 2.0 * nu;
        c[i] = 4.0 * (xi - 1.0) * (nu + xi - 1.0) * (nu + xi - 1.0) * (s + xi - 1.0) /
               ((s + 2.0 * xi - 1.0) * (s + 2.0 * xi - 2.0) * (s + 2.0 * xi - 2.0) * (s + 2.0 * xi - 3.0));
    }
    double cc = tsa;
    for (int i = 2; i <= n; ++i) cc *= c[i];
    auto eval = [&](double xv, double &pn, double &dpn, double &pn1) {
        double p1 = 1.0, p = xv, dp1 = 0.0, dp = 1.0;  // (alf-bta)/(alf+bta+2) = 0
        for (int j = 2; j <= n; ++j) {
            const double q = xv * p - c[j] * p1;
            const double dq = xv * dp + p - c[j] * dp1;
            p1 = p;
            p = q;
            dp1 = dp;
            dp = dq;
        }
        pn = p;
        dpn = dp;
        pn1 = p1;
    };
    const double step = (double)0.0001f, lim = (double)(-0.002f);
    std::vector<double> guess;
    double sgn = 1.0, xs = 1.0, p, dp, p1;
    for (;;) {
        eval(xs, p, dp, p1);
        if (sgn * p < 0.0) {
            sgn = -sgn;
            guess.push_back(xs);
        }
        if ((int)guess.size() == n2) break;
        xs -= step;
        if (!(xs > lim))
            raise(DVR3D_ERR_QUADRATURE, "Gauss-Jacobi scan found the wrong number of zeros");
    }
    x.assign(n2, 0.0);
    w.assign(n2, 0.0);
    csa = 0.0;
    for (int i = 0; i < n2; ++i) {
        double xr = guess[i], dpn = 0.0;
        for (int it = 1;; ++it) {
            eval(xr, p, dp, p1);
            const double d = p / dp;
            xr -= d;
            if (std::fabs(d) <= 1.0e-12 || it >= 10) break;
        }
        dpn = dp;
        x[i] = xr;
        w[i] = cc / (dpn * p1);
        csa += 2.0 * w[i];
    }
    if (2 * n2 != n) csa -= w[n2 - 1];
}

// Normalisation of the Laguerre basis (norms :1261-1287); also returns cc.
void laguerre_norms(int npnt, int nmax, double alf, std::vector<double> &dnorm, double &cc) {
    std::vector<double> fact(npnt + 2);
    fact[1] = 1.0;
    for (int i = 1; i <= npnt; ++i) fact[i + 1] = (double)i * fact[i];
    double count = (double)npnt + alf;
    cc = fact[npnt] / count;
    std::vector<double> bin(npnt + 2);
    bin[npnt + 1] = 1.0;
    for (int i = 1; i <= npnt; ++i) {
        bin[npnt + 1 - i] = bin[npnt + 2 - i] * count / (double)i;
        count -= 1.0;
    }
    dnorm.assign(nmax + 1, 0.0);
    for (int i = 0; i <= nmax; ++i) dnorm[i] = std::sqrt(bin[i + 1] * fact[i + 1] * fact[npnt + 1 - i]);
}

// One Morse radial coordinate: grid, weights, and DVR kinetic matrix (lagpt, keints, k1k2).
void morse_radial(int npnt, double re, double beta, double a, int iu, double ur,
                  std::vector<double> &y, std::vector<double> &wt, std::vector<double> &r,
                  std::vector<double> &xk, double &csx, double &csa, double &tsx, double &tsa) {
    const int nmax = npnt - 1;
    const double alf = (double)iu;
    std::vector<double> dnorm;
    double cc;
    laguerre_norms(npnt, nmax, alf, dnorm, cc);
    gauss_laguerre(npnt, alf, cc, y, wt, csx, csa, tsx);
    tsa = 1.0 / (dnorm[0] * dnorm[0]);
    if (std::fabs((csx - tsx) / tsx) > 1.0e-8 || std::fabs((csa - tsa) / tsa) > 1.0e-8)
        raise(DVR3D_ERR_QUADRATURE, "Gauss-Laguerre points & weights in error");
    r.assign(npnt, 0.0);
    // normalised Laguerre functions at the points: basis(n, i)
    std::vector<double> basis((size_t)npnt * (nmax + 1));
    for (int i = 0; i < npnt; ++i) {
        r[i] = re + std::log(a / y[i]) / beta;
        double *bs = &basis[(size_t)i * (nmax + 1)];
        bs[0] = 1.0;
        if (nmax >= 1) {
            double amx = alf + 1.0 - y[i], en = 1.0;
            bs[1] = amx;
            for (int n = 2; n <= nmax; ++n) {
                en += 1.0;
                amx += 2.0;
                bs[n] = (amx * bs[n - 1] - (alf - 1.0 + en) * bs[n - 2]) / en;
            }
        }
        for (int n = 0; n <= nmax; ++n) bs[n] *= dnorm[n];
    }
    // analytic Morse kinetic energy in the FBR, packed triangle (keints)
    const double fke = beta * beta / (8.0 * ur);
    auto hfbr = [&](int m, int mp) -> double {
        int lo = std::min(m, mp), hi = std::max(m, mp);  // 0-based orders
        if (lo == hi) return fke * (double)(2 * hi * (hi + 1 + iu) + iu + 1);
        if (lo + 2 == hi) {
            const int n1 = lo + 1;
            return -fke * std::sqrt((double)((long long)(iu + n1 + 1) * (iu + n1)) * (double)((n1 + 1) * n1));
        }
        return 0.0;
    };
    std::vector<double> hb((size_t)(nmax + 1) * (nmax + 1));
    for (int m = 0; m <= nmax; ++m)
        for (int mp = 0; mp <= nmax; ++mp) hb[(size_t)m * (nmax + 1) + mp] = hfbr(m, mp);
    // DVR transform xk(k,k') = sqrt(w_k w_k') sum_{m,m'} B(m,k) h(m,m') B(m',k') (k1k2)
    std::vector<double> sw(npnt);
    for (int i = 0; i < npnt; ++i) sw[i] = std::sqrt(wt[i]);
    xk.assign((size_t)npnt * npnt, 0.0);
    for (int k = 0; k < npnt; ++k) {
        const double *bk = &basis[(size_t)k * (nmax + 1)];
        for (int kp = 0; kp <= k; ++kp) {
            const double *bkp = &basis[(size_t)kp * (nmax + 1)];
            const double wkk = sw[k] * sw[kp];
            double acc = 0.0;
            for (int m = 0; m <= nmax; ++m) {
                const double t = bk[m] * wkk;
                const double *hrow = &hb[(size_t)m * (nmax + 1)];
                for (int mp = 0; mp <= nmax; ++mp) acc += hrow[mp] * t * bkp[mp];
            }
            xk[(size_t)kp * npnt + k] = acc;
            xk[(size_t)k * npnt + kp] = acc;
        }
    }
}

}  // namespace

void k_range(const dvr3d_deck &d, int &kd, int &ku) {
    int jrot = std::abs(d.jrot), kmin = d.kmin;
    bool zrot = d.zrot && jrot != 0;
    if (jrot == 0) kmin = 0;
    if (d.zperp && d.idia == -2) kmin = (jrot == 0) ? 0 : 1;  // KMIN is the Q symmetry (:257-261)
    if (zrot) {
        bool zbisc = (d.idia == -2);
        if (kmin != 0 && !zbisc) kmin = 1;
        if (kmin != 0 && kmin != 1) kmin = 2;
        kd = 1 - std::min(kmin, 1);
        ku = jrot + (kmin == 2 ? 1 : 0);
    } else {
        kd = ku = kmin;
    }
}

void plan_block(const dvr3d_deck &d, int kk, BlockPlan &p) {
    p = BlockPlan();
    if (d.ztwod) raise(DVR3D_ERR_UNSUPPORTED, "ztwod (fixed-angle 2D) is not on this path");
    if (d.zperp && d.idia == 2) raise(DVR3D_ERR_ARG, "ZPERP is for Radau coordinates (IDIA = -2), not IDIA = 2");
    if (d.ncoord == 2) raise(DVR3D_ERR_UNSUPPORTED, "ncoord=2 (rigid diatom) is not on this path");
    if (!d.zquad2) raise(DVR3D_ERR_UNSUPPORTED, "zquad2=F is not on this path");
    if (!d.zmors1 || !d.zmors2) raise(DVR3D_ERR_UNSUPPORTED, "spherical oscillators (zmors=F) are not on this path");
    if (d.zs0 || d.zs1) raise(DVR3D_ERR_UNSUPPORTED, "zs0/zs1 NBO corrections are not on this path");
    int npnt1 = d.npnt1, npnt2 = d.npnt2, nalf = d.nalf, jrot = d.jrot, kmin = d.kmin;
    int idia = d.idia, ipar = d.ipar, max2d = d.max2d, max3d = d.max3d, max3d2 = d.max3d2;
    int neval = d.neval;
    bool zrot = d.zrot, zembed = d.zembed, ztheta = d.ztheta, zall = d.zall, zbisc = false;
    if (idia != 1 && idia != 2 && idia != -1 && idia != -2) raise(DVR3D_ERR_ARG, "IDIA must be 1, 2, -1 or -2");
    // insize :241-264
    if (jrot == 0) {
        zembed = true;
        kmin = 0;
        zrot = false;
    }
    int idvr = nalf;
    const bool zperp = d.zperp != 0;
    int iq = 0;
    if (idia == -2) {
        npnt1 = npnt2;
        ztheta = false;
        if (jrot != 0) zbisc = true;
        if (zperp) {  // Q symmetry from the KMIN card field, k from 0 (:255-261)
            iq = kmin;
            kmin = (jrot == 0) ? 0 : 1;
        }
    }
    // the z-perp angular grid holds 2 nang2 Gauss-Jacobi points in an array of nalf (:945):
    // an odd nalf, or a later k block with fewer angles (zladd = F), would read points the
    // reference leaves undefined
    if (zperp && (idia != -2 || (nalf & 1) || !d.zladd))
        raise(DVR3D_ERR_UNSUPPORTED, "zperp needs IDIA = -2, an even NALF and ZLADD = T");
    if (npnt1 < 2 || npnt2 < 2 || nalf < 2 || npnt1 > 120 || npnt2 > 120 || nalf > 250)
        raise(DVR3D_ERR_ARG, "grid sizes out of range (2..120 radial, 2..250 angular)");
    const int nalf2 = (nalf + 1) / 2;
    const int mi = std::max(1, idia);
    int npnta, npntb, npntc;
    if (ztheta) {
        npnta = nalf / mi;
        npntb = d.zr2r1 ? npnt2 : npnt1;
        npntc = d.zr2r1 ? npnt1 : npnt2;
    } else {
        npnta = d.zr2r1 ? npnt2 : npnt1;
        npntb = d.zr2r1 ? npnt1 : npnt2;
        npntc = nalf / mi;
    }
    int max2d2 = 0;
    if (idia == -2) {
        if (zrot && (jrot + kmin) > 1) {
            max2d = npnt1 * (npnt1 + 1) / 2;
            max2d2 = npnt1 * (npnt1 - 1) / 2;
        } else {
            max2d = npnt1 * (npnt1 + 1 - ipar * 2) / 2;
        }
        max3d = zall ? max2d * nalf : std::min(max3d, max2d * nalf);
        if (zrot) {
            if (max3d2 <= 0) max3d2 = max3d;
            max3d2 = std::min(std::min(max3d, max2d2 * nalf), max3d2);
        }
    } else if (zall) {
        max2d = npnta * npntb;
        max3d = max2d * npntc;
    } else {
        max2d = std::min(max2d, npnta * npntb);
        max3d = std::min(max3d, npnta * npntb * npntc);
    }
    if (neval <= 0) neval = 10;
    neval = std::min(max3d, neval);
    if (std::abs(idia) == 2) {
        if (ipar != 0 && ipar != 1) raise(DVR3D_ERR_ARG, "illegal value of ipar for idia = +/-2");
        if (idia == 2) {
            idvr = nalf2;
            if (2 * idvr != nalf) raise(DVR3D_ERR_ARG, "nalf must be even when idia=2");
        }
    } else {
        ipar = 0;
    }
    if (jrot != 0) {
        jrot = std::abs(jrot);
        if (zrot) {
            if (kmin != 0 && !zbisc) kmin = 1;
            if (kmin != 0 && kmin != 1) kmin = 2;
        } else if (std::abs(kmin) > jrot) {
            raise(DVR3D_ERR_ARG, "k greater than J");
        }
        if (zbisc) zembed = false;
    }
    if (max3d <= 0 || (idia != -2 && max2d <= 0)) raise(DVR3D_ERR_ARG, "MAX2D/MAX3D must be positive");

    // setcon :1070-1125, :1144-1148
    double xm[3], xr[3];
    for (int i = 0; i < 3; ++i) {
        xm[i] = d.xmass[i];
        xr[i] = d.xmassr[i];
        if (xm[i] <= 0.0) raise(DVR3D_ERR_ARG, "masses must be positive");
    }
    if (xr[0] <= 0.0)
        for (int i = 0; i < 3; ++i) xr[i] = xm[i];
    if (idia >= 1) {
        p.g1 = xm[1] / (xm[1] + xm[2]);
        p.g2 = 0.0;
    } else {
        const double a = std::sqrt(xm[2] / (xm[0] + xm[1] + xm[2]));
        const double b = xm[1] / (xm[0] + xm[1]);
        p.g1 = 1.0 - a / (a + b - a * b);
        p.g2 = 1.0 - a / (1.0 - b + a * b);
    }
    auto redmass = [](double g, const double *m, bool first) {
        return first ? kAmToAu / (g * g / m[0] + 1.0 / m[1] + (1.0 - g) * (1.0 - g) / m[2])
                     : kAmToAu / (1.0 / m[0] + g * g / m[1] + (1.0 - g) * (1.0 - g) / m[2]);
    };
    p.ur1 = redmass(p.g2, xm, true);
    p.ur2 = redmass(p.g1, xm, false);
    p.urr1 = redmass(p.g2, xr, true);
    p.urr2 = redmass(p.g1, xr, false);
    if (d.diss1 <= 0.0 || d.we1 <= 0.0) raise(DVR3D_ERR_ARG, "r1 Morse parameters must be positive");
    p.beta1 = d.we1 * std::sqrt(0.5 * p.ur1 / d.diss1);
    p.a1 = 4.0 * d.diss1 / d.we1;
    p.iu1 = (int)(p.a1 + 0.5);
    if (idia != -2) {
        if (d.diss2 <= 0.0 || d.we2 <= 0.0) raise(DVR3D_ERR_ARG, "r2 Morse parameters must be positive");
        p.beta2 = d.we2 * std::sqrt(0.5 * p.ur2 / d.diss2);
        p.a2 = 4.0 * d.diss2 / d.we2;
        p.iu2 = (int)(p.a2 + 0.5);
    }
    // radial grids and kinetic matrices (ccmain :764-804)
    morse_radial(npnt1, d.re1, p.beta1, p.a1, p.iu1, p.ur1, p.y1, p.w1, p.r1, p.xk1, p.csx1,
                 p.csa1, p.tsx1, p.tsa1);
    if (idia > -2)
        morse_radial(npnt2, d.re2, p.beta2, p.a2, p.iu2, p.ur2, p.y2, p.w2, p.r2, p.xk2,
                     p.csx2, p.csa2, p.tsx2, p.tsa2);
    else
        p.r2 = p.r1;

    // replay the k loop up to kk (ccmain :811-998)
    int kd, ku;
    if (zrot) {
        kd = 1 - std::min(kmin, 1);
        ku = jrot + (kmin == 2 ? 1 : 0);
    } else {
        kd = ku = kmin;
    }
    if (kk < kd || kk > ku) raise(DVR3D_ERR_ARG, "k block index outside the k loop of this deck");
    const int max2d1 = max2d, max3d1 = max3d;
    int kz = 0, lincr = 0, nidvr = idvr, nang = nalf, nang2 = nalf2, kkz0 = 0, kkz12 = 0;
    for (int k = kd; k <= kk; ++k) {
        if (k <= jrot) {
            kz = k;
        } else {
            kz = 1;
            kmin = 0;
            if (!zperp) ipar = (ipar + jrot) % 2;
        }
        if (d.zladd || kz == kd) {
            nidvr = idvr;
            nang = nalf;
            nang2 = nalf2;
            lincr = kz;
        } else {
            lincr = 0;
            if (idia != 2) {
                nidvr = idvr - kz;
                nang = nalf - kz;
            } else if (ipar == 0) {
                if (kz % 2 == 1) kkz0 += 2;
                nidvr = idvr - kkz0 / 2;
                nang = nalf - kkz0;
            } else {
                if (kz % 2 == 0 && kz > 0) kkz12 += 2;
                nidvr = idvr - kkz12 / 2;
                nang = nalf - kkz12;
            }
            nang2 = (nang + 1) / 2;
        }
        if (!d.zladd) {
            if (ztheta) npnta = nidvr;
            else npntc = nidvr;
        }
        if (idia <= -2 && zrot) {
            if (kz > kd && !zperp) ipar = (ipar + 1) % 2;
            max2d = ipar > 0 ? max2d2 : max2d1;
            max3d = ipar > 0 ? max3d2 : max3d1;
        }
    }
    const int maxleg = nalf - 1;
    if (zperp) {
        // Gauss-Jacobi points with alpha = beta = sqrt((J(J+1) - k^2)/2), normalised Jacobi
        // polynomials, square-rooted weights (ccmain :945-966); L matrix with the weights
        // (j+1+alpha)(j+alpha) from j = 0 (lmatrx :1870-1903)
        const double rj = jrot, rk = kz;
        p.alf = std::sqrt(0.5 * ((rj * rj + rj) - rk * rk));
        std::vector<double> xg, wg;
        gauss_jacobi_full(2 * nang2, p.alf, p.alf, xg, wg);
        p.xalf.assign(idvr, 0.0);
        p.walf.assign(idvr, 0.0);
        for (int i = 0; i < idvr && i < (int)xg.size(); ++i) {
            p.xalf[i] = xg[i];
            p.walf[i] = std::sqrt(wg[i]);
        }
        p.whalf.assign(wg.begin(), wg.begin() + nang2);
        p.xhalf.assign(xg.begin(), xg.begin() + nang2);
        const std::vector<double> pj = jacobi_poly_basis(p.xalf, nidvr, maxleg, p.alf, p.alf);
        p.pleg_walf.assign((size_t)(maxleg + 1) * nidvr, 0.0);
        for (int i = 0; i < nidvr; ++i)
            for (int l = 0; l <= maxleg; ++l)
                p.pleg_walf[(size_t)i * (maxleg + 1) + l] = pj[(size_t)i * (maxleg + 1) + l] * p.walf[i];
        p.xlmatr.assign((size_t)idvr * idvr, 0.0);
        for (int k = 0; k < nidvr; ++k)
            for (int kp = k; kp < nidvr; ++kp) {
                double sum = 0.0;
                for (int j = 0; j <= maxleg; ++j)
                    sum += pj[(size_t)k * (maxleg + 1) + j] * pj[(size_t)kp * (maxleg + 1) + j] *
                           ((j + 1 + p.alf) * (j + p.alf));
                const double v = sum * p.walf[k] * p.walf[kp];
                p.xlmatr[(size_t)k * idvr + kp] = v;
                p.xlmatr[(size_t)kp * idvr + k] = v;
            }
    } else {
        // Gauss-(associated) Legendre points (:887-944) and allpts (:1747-1772)
        double tswalf = std::pow(2.0, kz + kz + 1) / (double)(kz + 1);
        for (int ia = 1; ia <= kz; ++ia) tswalf = tswalf * (double)ia / (double)(kz + ia + 1);
        gauss_jacobi_half(nang, nang2, (double)kz, tswalf, p.xhalf, p.whalf, p.cswalf);
        p.tswalf = tswalf;
        if (std::fabs((p.cswalf - tswalf) / tswalf) > 1.0e-8)
            raise(DVR3D_ERR_QUADRATURE, "Gauss-Legendre points & weights in error");
        p.xalf.assign(idvr, 0.0);
        p.walf.assign(idvr, 0.0);
        const double scale = (double)std::max(1, idia);
        for (int i = 0; i < nang2; ++i) {
            const double wv = std::sqrt(scale * p.whalf[i]);
            if (idia == 2) {
                p.xalf[i] = p.xhalf[i];
                p.walf[i] = wv;
            } else {
                p.xalf[nang - 1 - i] = p.xhalf[i];
                p.walf[nang - 1 - i] = wv;
                p.xalf[i] = -p.xhalf[i];
                p.walf[i] = wv;
            }
        }
        // normalised associated Legendre polynomial parts (asleg :1775-1843)
        const int m = kz;
        const int nl = maxleg + lincr - m + 1;  // orders j = m .. maxleg+lincr
        std::vector<double> pl((size_t)std::max(nl, 2) * nidvr, 0.0);
        for (int i = 0; i < nidvr; ++i) {
            double pmm = 1.0, f = 1.0;
            for (int j = 1; j <= m; ++j) {
                pmm = -pmm * f;
                f += 2.0;
            }
            double *col = &pl[(size_t)i * std::max(nl, 2)];
            col[0] = pmm;
            double pmmp1 = p.xalf[i] * (m + m + 1) * pmm;
            col[1] = pmmp1;
            int ll = 1;
            for (int l = 2 + m; l <= maxleg + lincr; ++l) {
                const double pll = (p.xalf[i] * (double)(l + l - 1) * pmmp1 - (double)(l + m - 1) * pmm) / (double)(l - m);
                pmm = pmmp1;
                pmmp1 = pll;
                col[++ll] = pll;
            }
        }
        std::vector<double> pnorm(std::max(nl, 1));
        for (int j = m, jj = 0; j <= maxleg + lincr; ++j, ++jj) {
            double f = 1.0;
            for (int i = j - m + 1; i <= j + m; ++i) f *= (double)i;
            pnorm[jj] = std::sqrt(((double)j + (double)j + 1.0) / (f + f));
        }
        for (int i = 0; i < nidvr; ++i)
            for (int jj = 0; jj < nl; ++jj) pl[(size_t)i * std::max(nl, 2) + jj] *= pnorm[jj];
        p.pleg_walf.assign((size_t)(maxleg + 1) * nidvr, 0.0);
        for (int i = 0; i < nidvr; ++i)
            for (int jj = 0; jj <= maxleg && jj < nl; ++jj)
                p.pleg_walf[(size_t)i * (maxleg + 1) + jj] = pl[(size_t)i * std::max(nl, 2) + jj] * p.walf[i];
        // angular kinetic matrix L(k,k') (lmatrx :1846-1911, in-plane)
        const int jdia = std::max(1, idia);
        const int ipar0 = (idia == 2 && ipar == 1) ? 1 : 0;
        int jstart = kz, jj0 = -jdia;
        if (jstart % jdia != ipar0) {
            ++jj0;
            ++jstart;
        }
        p.xlmatr.assign((size_t)idvr * idvr, 0.0);
        const int ld = std::max(nl, 2);
        for (int k = 0; k < nidvr; ++k) {
            for (int kp = k; kp < nidvr; ++kp) {
                double s = 0.0;
                int jj = jj0;
                for (int j = jstart; j <= maxleg + lincr; j += jdia) {
                    jj += jdia;
                    s += pl[(size_t)k * ld + jj] * pl[(size_t)kp * ld + jj] * (double)((j + 1) * j);
                }
                const double v = s * p.walf[k] * p.walf[kp];
                p.xlmatr[(size_t)k * idvr + kp] = v;
                p.xlmatr[(size_t)kp * idvr + k] = v;
            }
        }
    }
    // J > 0 angular-momentum terms
    p.term = (double)(jrot * jrot + jrot - 2 * kz * kz);  // jhmain :1970
    p.xp0 = d.zx ? 1.0 : 0.0;
    if (jrot != 0 && zperp) {  // z_blc2d1 :4059-4073
        const double rj = jrot, rk = kz;
        p.nf_term = rk * rk / 4.0;                                           // k^2 / 4
        p.nf_term2 = (1.0 - p.urr1 / p.ur1) * (rj * rj + rj - rk * rk) / 4.0;  // s (J(J+1) - k^2) / 4
        p.nf_term3 = (iq == 0) ? -rj * (rj + 1.0) / 4.0 : rj * (rj + 1.0) / 4.0;
    } else if (jrot != 0) {  // nfmain :3057-3064
        p.nf_term = (double)(jrot * jrot + jrot - kz * kz) / 8.0;
        p.nf_term2 = (double)(jrot * jrot + jrot - 3 * kz * kz) / 4.0;
        if (std::abs(kz) == 1) {
            p.nf_term3 = (double)(jrot * jrot + jrot) / 16.0;
            if (kmin >= 1 && zrot) p.nf_term3 = -p.nf_term3;
        }
    }
    p.npnt1 = npnt1;
    p.npnt2 = npnt2;
    p.nalf = nalf;
    p.idvr = idvr;
    p.nidvr = nidvr;
    p.maxleg = maxleg;
    p.neval = neval;
    p.jrot = jrot;
    p.kmin = kmin;
    p.idia = idia;
    p.ipar = ipar;
    p.kz = kz;
    p.kd = kd;
    p.ku = ku;
    p.lincr = lincr;
    p.max2d = max2d;
    p.max3d = max3d;
    p.npnta = npnta;
    p.npntb = npntb;
    p.npntc = npntc;
    p.radau = (idia == -2);
    p.zperp = zperp;
    p.iq = iq;
    p.ztheta = ztheta;
    p.zr2r1 = d.zr2r1;
    p.zcut = d.zcut || zall;
    p.zall = zall;
    p.zembed = zembed;
    p.zlin = d.zlin;
    p.zrot = zrot;
    p.emax1_au = d.emax1 / kAuToCm;
    p.emax2_au = d.emax2 / kAuToCm;
}

}  // namespace dvr3d
