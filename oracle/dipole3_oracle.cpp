// dipole3_oracle.cpp -- CPU restatement of the reference's program DIPOLE3
// (source/dipole3_segmented.f90): transition moments between the vib-rot states of two
// wavefunction files (ket: unit IKET = 11, bra: unit IBRA = 12) on a user dipole surface, the
// printed table of spect and the ITRA (fort.13) records of outpt.
//
// TEST INFRASTRUCTURE ONLY: the parity checker of the product's dvr3d_b200_dipole3. It follows
// the reference routine by routine, reading both files record by record as the reference does
// (its k-block record counting, the bra blocks kept for k-1, k, k+1), with the rank-1 updates of
// trans as loops. Nothing in the product links or calls it.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../include/dvr3d_b200.h"
#include "dvr3d_oracle.h"

namespace {

struct DFail {
    int code;
};
[[noreturn]] void dfail(int code) { throw DFail{code}; }

// A sequential unformatted file: records framed by 4-byte lengths, read in order, rewound.
struct SeqFile {
    std::vector<unsigned char> b;
    std::vector<std::pair<size_t, size_t>> recs;
    size_t next = 0;
    explicit SeqFile(const char *path) {
        FILE *fp = std::fopen(path, "rb");
        if (!fp) dfail(DVR3D_ERR_ARG);
        std::fseek(fp, 0, SEEK_END);
        const long n = std::ftell(fp);
        std::fseek(fp, 0, SEEK_SET);
        b.resize((size_t)n);
        const size_t got = n > 0 ? std::fread(b.data(), 1, (size_t)n, fp) : 0;
        std::fclose(fp);
        if (got != (size_t)n) dfail(DVR3D_ERR_ARG);
        size_t p = 0;
        while (p + 8 <= b.size()) {
            int32_t m;
            std::memcpy(&m, &b[p], 4);
            if (m < 0 || p + 8 + (size_t)m > b.size()) dfail(DVR3D_ERR_ARG);
            recs.emplace_back(p + 4, (size_t)m);
            p += 8 + (size_t)m;
        }
    }
    void rewind() { next = 0; }
    std::pair<const unsigned char *, size_t> rec() {
        if (next >= recs.size()) dfail(DVR3D_ERR_ARG);  // end of file
        auto r = recs[next++];
        return {&b[r.first], r.second};
    }
    void skip() { rec(); }
    std::vector<int> ints(size_t n) {
        auto r = rec();
        if (r.second < 4 * n) dfail(DVR3D_ERR_ARG);
        std::vector<int> v(n);
        std::memcpy(v.data(), r.first, 4 * n);
        return v;
    }
    // read(iu) (dum, i = 1, nskip), row(1:n)
    void getrow(double *row, size_t n, size_t nskip = 0) {
        auto r = rec();
        if (r.second < 8 * (n + nskip)) dfail(DVR3D_ERR_ARG);
        std::memcpy(row, r.first + 8 * nskip, 8 * n);
    }
};

bool lg(const unsigned char *p) {
    int32_t v;
    std::memcpy(&v, p, 4);
    return v != 0;
}
double r8(const unsigned char *p) {
    double v;
    std::memcpy(&v, p, 8);
    return v;
}

struct Header {
    int idia, ipar, lmax, nmax1, nmax2, jrot, kmin, neval;
    bool zemb, zmor1, zmor2, znco;
    double xm[3], g1, g2;
};

Header read_header(SeqFile &f) {
    Header h{};
    std::vector<int> a = f.ints(8);
    h.idia = a[0];
    h.ipar = a[1];
    h.lmax = a[2];
    h.nmax1 = a[3];
    h.nmax2 = a[4];
    h.jrot = a[5];
    h.kmin = a[6];
    h.neval = a[7];
    auto r = f.rec();
    if (r.second < 56) dfail(DVR3D_ERR_ARG);
    h.zemb = lg(r.first);
    h.zmor1 = lg(r.first + 4);
    h.zmor2 = lg(r.first + 8);
    for (int i = 0; i < 3; ++i) h.xm[i] = r8(r.first + 12 + 8 * i);
    h.g1 = r8(r.first + 36);
    h.g2 = r8(r.first + 44);
    h.znco = lg(r.first + 52);
    return h;
}

// ---- the job deck: namelist PRT, title (9a8), npot nv1 nv2 ibase1 ibase2 (5i5), ezero (f20.0)
struct DipDeck {
    bool zprint = false, zpmin = false, ztra = true, zstart = false;
    int ires = 0, nblock = 1000;
    std::string title;
    int npot = 0, nv1 = 0, nv2 = 0, ibase1 = 0, ibase2 = 0;
    double ezero = 0.0;
    bool have_ezero = false;
};

std::string lower(std::string s) {
    for (auto &c : s) c = (char)std::tolower((unsigned char)c);
    return s;
}

DipDeck parse_dip_deck(const char *text) {
    std::vector<std::string> lines;
    std::string cur;
    for (const char *c = text; *c; ++c) {
        if (*c == '\n') {
            lines.push_back(cur);
            cur.clear();
        } else if (*c != '\r') {
            cur += *c;
        }
    }
    if (!cur.empty()) lines.push_back(cur);
    DipDeck d;
    size_t i = 0;
    while (i < lines.size() && lines[i].find('&') == std::string::npos) ++i;
    if (i == lines.size()) dfail(DVR3D_ERR_DECK);
    std::string nl;
    for (; i < lines.size(); ++i) {
        nl += lines[i] + " ";
        if (lines[i].find('/') != std::string::npos) break;
    }
    if (i == lines.size()) dfail(DVR3D_ERR_DECK);
    ++i;
    nl = lower(nl);
    nl = nl.substr(nl.find('&') + 1);
    nl = nl.substr(0, nl.find('/'));
    size_t p = nl.find_first_of(" \t,");
    nl = p == std::string::npos ? std::string() : nl.substr(p);  // drop the group name
    for (auto &c : nl)
        if (c == ',') c = ' ';
    // key = value pairs
    size_t q = 0;
    while (q < nl.size()) {
        size_t e = nl.find('=', q);
        if (e == std::string::npos) break;
        std::string key = nl.substr(q, e - q);
        key.erase(0, key.find_first_not_of(" \t"));
        key.erase(key.find_last_not_of(" \t") + 1);
        size_t vb = nl.find_first_not_of(" \t", e + 1);
        if (vb == std::string::npos) break;
        size_t ve = nl.find_first_of(" \t", vb);
        std::string val = nl.substr(vb, ve == std::string::npos ? std::string::npos : ve - vb);
        q = ve == std::string::npos ? nl.size() : ve;
        auto logical = [&]() {
            std::string v = val;
            if (!v.empty() && v[0] == '.') v = v.substr(1);
            return !v.empty() && v[0] == 't';
        };
        if (key == "zprint") d.zprint = logical();
        else if (key == "zpmin") d.zpmin = logical();
        else if (key == "ztra") d.ztra = logical();
        else if (key == "zstart") d.zstart = logical();
        else if (key == "ires") d.ires = std::atoi(val.c_str());
        else if (key == "nblock") d.nblock = std::atoi(val.c_str());
    }
    if (i < lines.size()) d.title = lines[i++].substr(0, 72);
    if (i >= lines.size()) dfail(DVR3D_ERR_DECK);
    auto i5 = [&](const std::string &s, int f) {
        if ((size_t)(5 * f) >= s.size()) return 0;
        std::string t = s.substr(5 * f, 5);
        size_t a = t.find_first_not_of(' ');
        return a == std::string::npos ? 0 : std::atoi(t.c_str() + a);
    };
    d.npot = i5(lines[i], 0);
    d.nv1 = i5(lines[i], 1);
    d.nv2 = i5(lines[i], 2);
    d.ibase1 = i5(lines[i], 3);
    d.ibase2 = i5(lines[i], 4);
    ++i;
    if (i < lines.size()) {  // read(5,505,end=555) ezero, f20.0
        std::string t = lines[i].substr(0, std::min<size_t>(20, lines[i].size()));
        for (auto &c : t)
            if (c == 'd' || c == 'D') c = 'e';
        if (t.find_first_not_of(' ') != std::string::npos) d.ezero = std::atof(t.c_str());
        d.have_ezero = true;
    }
    return d;
}

// ---- quadrature and angular functions
// recur :1389-1410
void drecur(double &pn, double &dpn, double &pn1, double x, int nn, double alf, double bta,
            const std::vector<double> &b, const std::vector<double> &c) {
    double p1 = 1.0, p = x + (alf - bta) / (alf + bta + 2.0), dp1 = 0.0, dp = 1.0;
    for (int j = 2; j <= nn; ++j) {
        const double q = (x - b[j]) * p - c[j] * p1;
        const double dq = (x - b[j]) * dp + p - c[j] * dp1;
        p1 = p;
        p = q;
        dp1 = dp;
        dp = dq;
    }
    pn = p;
    dpn = dp;
    pn1 = p1;
}

// root :1370-1387
void droot(double &x, int nn, double alf, double bta, double &dpn, double &pn1, const std::vector<double> &b,
           const std::vector<double> &c, double eps) {
    int iter = 0;
    double p, dp;
    for (;;) {
        ++iter;
        drecur(p, dp, pn1, x, nn, alf, bta, b, c);
        const double d = p / dp;
        x = x - d;
        if (!(std::fabs(d) > eps && iter < 10)) break;
    }
    dpn = dp;
}

// jacobi :1311-1368 (Stroud and Secrest's starting values; REAL*4 literals kept as such)
void djacobi(int nn, std::vector<double> &x, std::vector<double> &a, double alf, double bta,
             const std::vector<double> &b, const std::vector<double> &c, double &csa, double &tsa) {
    const double eps = 1.0e-12, fn = (double)nn;
    const int nn2 = nn / 2;
    csa = 0.0;
    double beta = 1.0;
    if (alf == 1) beta = beta / 6.0;
    double cc = beta * std::pow(2.0, alf + bta + 1.0);
    tsa = cc / 2.0;
    for (int i = 2; i <= nn; ++i) cc = cc * c[i];
    double xt = 0.0;
    for (int i = 1; i <= nn2; ++i) {
        if (i == 1) {
            const double an = alf / fn, bn = bta / fn;
            const double r1 = (1.0 + alf) * (2.78 / (4.0 + fn * fn) + (double)0.768f * an / fn);
            const double r2 = 1.0 + 1.48 * an + 0.96 * bn + (double)0.452f * an * an + 0.83 * an * bn;
            xt = 1.0 - r1 / r2;
        } else if (i == 2) {
            const double r1 = (4.1 + alf) / ((1.0 + alf) * (1.0 + (double)0.156f * alf));
            const double r2 = 1.0 + 0.06 * (fn - 8.0) * (1.0 + 0.12 * alf) / fn;
            const double r3 = 1.0 + (double)0.012f * bta * (1.0 + std::fabs(alf) / 4.0) / fn;
            xt = xt - r1 * r2 * r3 * (1.0 - xt);
        } else if (i == 3) {
            const double r1 = (1.67 + 0.28 * alf) / (1.0 + 0.37 * alf);
            const double r2 = 1.0 + 0.22 * (fn - 8.0) / fn;
            const double r3 = 1.0 + 8.0 * bta / ((6.28 + bta) * fn * fn);
            xt = xt - r1 * r2 * r3 * (x[1] - xt);
        } else {
            xt = 3.0 * x[i - 1] - 3.0 * x[i - 2] + x[i - 3];
        }
        double dpn, pn1;
        droot(xt, nn, alf, bta, dpn, pn1, b, c, eps);
        x[i] = xt;
        a[i] = cc / (dpn * pn1);
        csa = csa + a[i];
    }
}

// asleg :1234-1309: normalised associated Legendre functions (sin^m kept), pleg(i, 0:lmax)
void dasleg(std::vector<double> &pleg, int lmax, const std::vector<double> &x, int ipot, int m) {
    pleg.assign((size_t)ipot * (lmax + 2), 0.0);
    auto P = [&](int i, int l) -> double & { return pleg[(size_t)(i - 1) + (size_t)ipot * l]; };
    for (int i = 1; i <= ipot; ++i) {
        if (m < 0 || std::fabs(x[i]) > 1.0) dfail(DVR3D_ERR_ARG);
        double pmm = 1.0, fact = 1.0;
        const double somx2 = std::sqrt((1.0 - x[i]) * (1.0 + x[i]));
        for (int j = 1; j <= m; ++j) {
            pmm = -pmm * fact * somx2;
            fact = fact + 2.0;
        }
        P(i, 0) = pmm;
        double pmmp1 = x[i] * (double)(m + m + 1) * pmm;
        P(i, 1) = pmmp1;
        int ll = 1;
        for (int l = 2 + m; l <= lmax + m; ++l) {
            const double pll = (x[i] * (double)(l + l - 1) * pmmp1 - (double)(l + m - 1) * pmm) / (double)(l - m);
            pmm = pmmp1;
            pmmp1 = pll;
            ++ll;
            P(i, ll) = pll;
        }
    }
    std::vector<double> pnorm(lmax + 1);
    int jj = -1;
    for (int j = m; j <= lmax + m; ++j) {
        double fact = 1.0;
        for (int i = j - m + 1; i <= j + m; ++i) fact = fact * (double)i;
        ++jj;
        pnorm[jj] = std::sqrt((double)(j + j + 1) / (fact + fact));
    }
    for (jj = 0; jj <= lmax; ++jj)
        for (int i = 1; i <= ipot; ++i) P(i, jj) = P(i, jj) * pnorm[jj];
}

// setfac :1118-1139: binom(i+1, j+1) = i! / (j! (i-j)!)
std::vector<double> setfac(int nbin) {
    std::vector<double> bn((size_t)nbin * nbin, 0.0);
    auto B = [&](int i, int j) -> double & { return bn[(size_t)(i - 1) + (size_t)nbin * (j - 1)]; };
    B(1, 1) = 1.0;
    if (nbin >= 2) {
        B(2, 1) = 1.0;
        B(2, 2) = 1.0;
    }
    for (int i = 3; i <= nbin; ++i) {
        B(i, 1) = 1.0;
        B(i, i) = 1.0;
        for (int j = 2; j <= i - 1; ++j) B(i, j) = B(i - 1, j - 1) + B(i - 1, j);
    }
    return bn;
}

// threej :1778-1823 (Racah's formula on the binomial table)
double threej(int j1, int j2, int j3, int m1, int m2, int m3, const std::vector<double> &bn, int nbin) {
    auto B = [&](int i, int j) {
        if (i < 1 || j < 1 || i > nbin || j > nbin) dfail(DVR3D_ERR_ARG);
        return bn[(size_t)(i - 1) + (size_t)nbin * (j - 1)];
    };
    double t = 0.0;
    if (m1 + m2 + m3 != 0) return t;
    const int i1 = -j1 + j2 + j3 + 1;
    if (i1 <= 0) return t;
    const int i2 = j1 - j2 + j3 + 1;
    if (i2 <= 0) return t;
    const int i3 = j1 + j2 - j3 + 1;
    if (i3 <= 0) return t;
    const int k1 = j1 + m1 + 1;
    if (k1 <= 0) return t;
    const int k2 = j2 + m2 + 1;
    if (k2 <= 0) return t;
    const int k3 = j3 + m3 + 1;
    if (k3 <= 0) return t;
    const int l1 = j1 - m1 + 1;
    if (l1 <= 0) return t;
    const int l2 = j2 - m2 + 1;
    if (l2 <= 0) return t;
    const int l3 = j3 - m3 + 1;
    if (l3 <= 0) return t;
    const int n1 = -j1 - m2 + j3, n2 = m1 - j2 + j3, n3 = j1 - j2 + m3;
    const int imin = std::max(std::max(-n1, -n2), 0) + 1;
    const int imax = std::min(std::min(l1, k2), i3);
    if (imin > imax) return t;
    double sign = 1.0;
    for (int i = imin; i <= imax; ++i) {
        sign = -sign;
        t = t + sign * B(i1, n1 + i) * B(i2, n2 + i) * B(i3, i);
    }
    t = t * std::sqrt(B(j2 + j2 + 1, i3) * B(j1 + j1 + 1, i2) /
                      (B(j1 + j2 + j3 + 2, i3) * (double)(j3 + j3 + 1) * B(j1 + j1 + 1, l1) * B(j2 + j2 + 1, l2) *
                       B(j3 + j3 + 1, l3)));
    if ((n3 + imin) % 2 != 0) t = -t;
    return t;
}

struct Dipole {
    dvr3d_dipd_fn dipd;
    dvr3d_dipsa_fn dipsa;
    void *user;
    double g1, g2;
    bool zembed, zbisc;
};

// DIPD :2054-2194, the reference's own coordinate transform around the user's DIPSA
double dipd_default(const Dipole &D, double r1, double r2, double xcos, int nu) {
    const double x1 = 1.0, x0 = 0.0, tiny = 9.0e-15, x2 = 2.0;
    const double g1 = D.g1, g2 = D.g2;
    double q1, q2, theta, cost = 0.0, beta = 0.0, alpha = 0.0;
    if (g1 == x0) {
        q1 = r1;
        q2 = r2;
        theta = std::acos(xcos);
        cost = xcos;
    } else if (g2 == x0) {
        const double xx = r1 * g1, yy = r1 * (x1 - g1);
        alpha = std::acos(xcos);
        if (r2 == x0 || xcos >= (x1 - tiny)) {
            q1 = std::fabs(xx - r2);
            q2 = (yy + r2);
            cost = -x1;
        } else if (xcos <= (tiny - x1)) {
            q1 = (xx + r2);
            q2 = std::fabs(yy + r2);
            cost = x1;
        } else {
            q1 = std::sqrt(xx * xx + r2 * r2 - x2 * xx * r2 * xcos);
            q2 = std::sqrt(yy * yy + r2 * r2 + x2 * yy * r2 * xcos);
            cost = (q1 * q1 + q2 * q2 - r1 * r1) / (x2 * q1 * q2);
        }
        const double xsin = std::sqrt(1.0 - xcos * xcos);
        theta = std::acos(cost);
        beta = std::asin(xsin * yy / q2);
    } else {
        const double f1 = x1 / g1, f2 = x1 / g2, f12 = x1 - f1 * f2;
        const double p1 = r1 * (x1 - f1) / (g2 * f12), p2 = r2 * (x1 - f2) / (g1 * f12);
        const double s1 = r1 - p1, s2 = r2 - p2;
        q1 = std::sqrt(p1 * p1 + s2 * s2 + x2 * p1 * s2 * xcos) / (x1 - g1);
        q2 = std::sqrt(p2 * p2 + s1 * s1 + x2 * p2 * s1 * xcos) / (x1 - g2);
        const double q3 = std::sqrt(p1 * p1 + p2 * p2 - x2 * p1 * p2 * xcos);
        cost = (q1 * q1 + q2 * q2 - q3 * q3) / (x2 * q1 * q2);
        theta = std::acos(cost);
    }
    double dipx = 0.0, dipy = 0.0;
    D.dipsa(&dipx, &dipy, q1, q2, cost, D.user);
    double dipc, ycos, ysin;
    if (g1 == x0) {
        const double gamma = theta / x2;
        ycos = std::cos(gamma);
        ysin = std::sin(gamma);
        if (D.zembed) dipc = nu == 0 ? dipy * ycos - dipx * ysin : dipx * ycos + dipy * ysin;
        else dipc = nu == 0 ? dipy * ycos + dipx * ysin : -dipx * ycos + dipy * ysin;
    } else if (g2 == x0) {
        const double gamma = beta - theta / x2;
        if (D.zembed) {
            ycos = std::cos(gamma);
            ysin = std::sin(gamma);
            dipc = nu == 0 ? -dipx * ysin - dipy * ycos : dipx * ycos - dipy * ysin;
        } else {
            const double delta = alpha - gamma;
            ycos = std::cos(delta);
            ysin = std::sin(delta);
            dipc = nu == 0 ? dipx * ysin + dipy * ycos : dipx * ycos - dipy * ysin;
        }
    } else {
        if (D.zbisc) {
            const double h1 = g1 * q1;
            const double cosa = (r2 * r2 + q2 * q2 - h1 * h1) / (x2 * r2 * q2);
            const double al = (std::acos(xcos) - theta) / x2 - std::acos(cosa);
            ycos = -std::cos(al);
            ysin = std::sin(al);
            dipc = nu == 1 ? dipx * ysin - dipy * ycos : -dipx * ycos - dipy * ysin;
        } else if (D.zembed) {
            const double h1 = g1 * q1;
            const double cosa = (r2 * r2 + h1 * h1 - q2 * q2) / (x2 * r2 * h1);
            const double al = std::acos(cosa);
            ycos = -std::cos(al + theta / x2);
            ysin = std::sin(al + theta / x2);
            dipc = nu == 0 ? -dipx * ysin + dipy * ycos : dipx * ycos + dipy * ysin;
        } else {
            const double h2 = g2 * q2;
            const double cosa = (r1 * r1 + h2 * h2 - q1 * q1) / (x2 * r1 * h2);
            const double al = std::acos(cosa);
            ycos = -std::cos(al + theta / x2);
            ysin = std::sin(al + theta / x2);
            dipc = nu == 0 ? dipx * ysin + dipy * ycos : -dipx * ycos + dipy * ysin;
        }
    }
    return dipc;
}

double call_dipd(const Dipole &D, double r1, double r2, double xcos, int nu) {
    return D.dipd ? D.dipd(r1, r2, xcos, nu, D.user) : dipd_default(D, r1, r2, xcos, nu);
}

std::string fmt_fd(double v, int w, int d, char ech = 'D') {  // Fortran Dw.d (Ew.d with ech = 'E')
    char buf[64];
    if (v == 0.0) {
        std::snprintf(buf, sizeof(buf), "0.%0*d%c+00", d, 0, ech);
    } else {
        int ex = (int)std::floor(std::log10(std::fabs(v))) + 1;
        const double scale = std::pow(10.0, d);
        double rm = std::round(std::fabs(v) / std::pow(10.0, ex) * scale);
        if (rm >= scale) {
            rm /= 10.0;
            ex += 1;
        }
        if (rm < scale / 10.0) {
            rm *= 10.0;
            ex -= 1;
        }
        std::snprintf(buf, sizeof(buf), "%s0.%0*.0f%c%c%02d", v < 0 ? "-" : "", d, rm, ech, ex < 0 ? '-' : '+',
                      std::abs(ex));
    }
    std::string s(buf);
    if ((int)s.size() < w) s = std::string(w - s.size(), ' ') + s;
    return s;
}

std::string fmt_es(double v, int w, int d) {  // Fortran ESw.d
    char buf[64];
    std::snprintf(buf, sizeof(buf), "%.*E", d, v);
    std::string s(buf);
    // C prints at least two exponent digits, as ES does below |exponent| 100
    if ((int)s.size() < w) s = std::string(w - s.size(), ' ') + s;
    return s;
}

struct Run {
    DipDeck dk;
    SeqFile *ket, *bra;
    Header h1, h2;
    int idia = 0, ipar1 = 0, ipar2 = 0, jrot1 = 0, jrot2 = 0, kmin1 = 0, kmin2 = 0;
    int npnt1 = 0, npnt2 = 0, nrade = 0, nrado = 0, mbass1 = 0, mbass2 = 0;
    int jk1 = 0, jk2 = 0, neval1 = 0, neval2 = 0, ibase1 = 1, ibase2 = 1;
    int npot = 0, nn2 = 0, ipot = 0, nbin = 0, mblock = 0, nblock = 0;
    bool zembed = false, zbisc = false, znco1 = false, znco2 = false;
    std::vector<int> nbass1, nbass2;
    std::vector<double> r1, r2, xd, wtd, dipol, binom;
    Dipole D{};
};

// genind :656-706
std::vector<int> genind(SeqFile &f, int mbass, int jk) {
    std::vector<int> a = f.ints(1 + 3 * (size_t)jk);
    if (a[0] > mbass) dfail(DVR3D_ERR_ARG);
    return std::vector<int>(a.begin() + 1 + 2 * jk, a.begin() + 1 + 3 * jk);
}

// lagpt :1141-1232: d0 = wtd * dipole at the radial DVR points and angular points
void lagpt(Run &R, int nu) {
    const int npot = R.npot;
    std::vector<double> b(npot + 1, 0.0), c(npot + 1, 0.0), x(npot + 1, 0.0), a(npot + 1, 0.0);
    const double alf = 0.0, bta = 0.0;
    for (int i = 2; i <= npot; ++i) {
        const double xi = (double)i;
        b[i] = (alf + bta) * (bta - alf) / ((alf + bta + 2.0 * xi) * (alf + bta + 2.0 * xi - 2.0));
        c[i] = 4.0 * (xi - 1.0) * (alf + xi - 1.0) * (bta + xi - 1.0) * (alf + bta + xi - 1.0) /
               ((alf + bta + 2.0 * xi - 1.0) * (alf + bta + 2.0 * xi - 2.0) * (alf + bta + 2.0 * xi - 2.0) *
                (alf + bta + 2.0 * xi - 3.0));
    }
    double csa, tsa;
    djacobi(npot, x, a, alf, bta, b, c, csa, tsa);
    if (std::fabs((csa - tsa) / tsa) > 1.0e-8) dfail(DVR3D_ERR_QUADRATURE);
    const int nn2 = R.nn2;
    for (int i = 1; i <= nn2; ++i) {
        if (R.idia >= 0) {
            const int j = i + nn2;
            x[j] = -x[npot - j + 1];
            a[j] = a[npot - j + 1];
        } else {
            const int j = npot + 1 - i;
            x[j] = -x[i];
            a[j] = a[i];
        }
    }
    R.xd = x;
    R.wtd = a;
    R.dipol.clear();
    const int jdia = std::max(1, R.idia);
    const int iadd = 1 - std::abs(nu);
    for (int i2 = 1; i2 <= R.npnt2; ++i2) {
        double rr2;
        int i0;
        if (R.idia == -2) {
            rr2 = R.r1[i2 - 1];
            i0 = i2 - iadd;
        } else {
            rr2 = R.r2[i2 - 1];
            i0 = R.npnt1;
        }
        for (int i1 = 1; i1 <= i0; ++i1)
            for (int j = 1; j <= R.ipot; ++j) {
                double v = call_dipd(R.D, R.r1[i1 - 1], rr2, x[j], nu);
                if (jdia == 2) v = 2.0 * v;
                R.dipol.push_back(a[j] * v);
            }
    }
}

// jtran :1564-1646 (J = 0 first-step files): coef(ne, nang*nrad) from the DVR amplitudes
void jtran(Run &R, SeqFile &f, std::vector<double> &coef, int nrad, int mvib, const std::vector<double> &pleg,
           int maxleg, int idvr, int kz, int ipar, const std::vector<int> &iv, int iang, int ibass, int ibase, int nu,
           int jay_ipar) {
    int jstart = kz;
    const int jdia = std::max(R.idia, 1);
    int jj0 = -jdia;
    if (R.zembed) {
        if (R.idia == 2 && jstart % 2 != R.ipar1) {
            ++jj0;
            ++jstart;
        }
    } else if (R.idia == 2 && jstart % 2 != jay_ipar) {
        ++jj0;
        ++jstart;
    }
    const int nang = (maxleg + kz - jstart) / jdia + 1;
    for (int l = 1; l <= ibase - 1; ++l) f.skip();
    coef.assign((size_t)mvib * nang * nrad, 0.0);
    std::vector<double> dvrvec((size_t)iang * std::max(nrad, R.nrade) + ibass, 0.0), temp(ibass);
    for (int l = 1; l <= mvib; ++l) {
        if (nu == 0 && R.idia == -2 && ipar == 0) {
            f.getrow(temp.data(), ibass);
            int ipt = 0, jpt = 0;
            for (int n1 = 1; n1 <= R.npnt1; ++n1) {
                for (int n2 = 1; n2 <= n1 - 1; ++n2) {
                    ++jpt;
                    ++ipt;
                    for (int j = 1; j <= iang; ++j) dvrvec[(j - 1) + (size_t)iang * (ipt - 1)] = temp[(j - 1) + (size_t)iang * (jpt - 1)];
                }
                ++jpt;
            }
        } else {
            f.getrow(dvrvec.data(), ibass);
        }
        int jj = jj0;
        for (int j = 1; j <= nang; ++j) {
            std::vector<double> sumk(nrad, 0.0);
            jj += jdia;
            int kk = 0;
            for (int k = 1; k <= idvr; ++k) {
                if (iv[k - 1] <= 0) continue;
                ++kk;
                for (int mn = 1; mn <= nrad; ++mn)
                    sumk[mn - 1] += dvrvec[(kk - 1) + (size_t)iang * (mn - 1)] * pleg[jj + (size_t)(maxleg + 1) * (k - 1)];
            }
            int ipt = j;
            for (int mn = 1; mn <= nrad; ++mn) {
                coef[(l - 1) + (size_t)mvib * (ipt - 1)] = sumk[mn - 1];
                ipt += nang;
            }
        }
    }
}

// dsrd :1412-1562: the vectors of one k block evaluated at the angular integration points,
// d(ne, nrad*ipot)
void dsrd(Run &R, std::vector<double> &d, SeqFile &f, int mmbass, int nbass, int ne, int kneed, int &kbeg, int jk,
          int ipar, int ibase, int kk, int nu, int jay_ipar) {
    int nang = nbass / R.nrade;
    if (ipar == 1 && R.zbisc) nang = nbass / R.nrado;
    int nrad = R.nrado;
    const int jdia = std::max(1, R.idia);
    if (std::abs(nu) == 1 && ipar == 0) nrad = R.nrade;
    std::vector<double> temp;  // temp(ne, nbass)
    int kz = 0;
    if (jk > 1) {
        kz = kk;
        if (kneed <= kbeg) {
            f.rewind();
            for (int i = 1; i <= kneed + 6; ++i) f.skip();
            if (!R.zbisc) f.skip();
        } else {
            for (int i = kbeg; i <= kneed - 2; ++i) f.skip();
        }
        // the record: (dum, nbass*(ibase-1)), ((d(i,j), j = 1, nbass), i = 1, ne)
        std::vector<double> rec((size_t)ne * nbass);
        f.getrow(rec.data(), (size_t)ne * nbass, (size_t)nbass * (ibase - 1));
        if (nang * nrad > nbass) dfail(DVR3D_ERR_ARG);
        temp.assign((size_t)ne * nbass, 0.0);
        if (nu == 0 && R.zbisc && ipar == 0) {
            int ipt = 0, jpt = 0;
            for (int n1 = 1; n1 <= R.npnt1; ++n1) {
                for (int n2 = 1; n2 <= n1 - 1; ++n2)
                    for (int j = 1; j <= nang; ++j) {
                        ++ipt;
                        ++jpt;
                        for (int ie = 1; ie <= ne; ++ie)
                            temp[(ie - 1) + (size_t)ne * (ipt - 1)] = rec[(jpt - 1) + (size_t)nbass * (ie - 1)];
                    }
                jpt += nang;
            }
        } else {
            for (int ie = 1; ie <= ne; ++ie)
                for (int j = 1; j <= nbass; ++j) temp[(ie - 1) + (size_t)ne * (j - 1)] = rec[(j - 1) + (size_t)nbass * (ie - 1)];
        }
    } else {
        f.rewind();
        for (int i = 1; i <= 6; ++i) f.skip();
        if (!R.zbisc) f.skip();
        std::vector<int> kh = f.ints(3);
        kz = kh[0];
        const int maxleg = kh[1], nidvr = kh[2];
        std::vector<double> plegd((size_t)(maxleg + 1) * nidvr);
        f.getrow(plegd.data(), plegd.size());
        int iang, ibass;
        std::vector<int> iv;
        if (R.zbisc) {
            std::vector<int> ib = f.ints(2);
            iang = ib[0];
            ibass = ib[1];
            iv = f.ints(nidvr);
        } else {
            iang = nidvr;
            ibass = mmbass;
            iv.assign(nidvr, 1);
        }
        f.skip();
        f.skip();
        if (iang <= 0 || ibass % iang != 0 || ibass / iang < nrad) dfail(DVR3D_ERR_ARG);
        jtran(R, f, temp, nrad, ne, plegd, maxleg, nidvr, kz, ipar, iv, iang, ibass, ibase, nu, jay_ipar);
    }
    if (nang < 1 || temp.size() < (size_t)ne * nrad * nang) dfail(DVR3D_ERR_ARG);
    std::vector<double> plegd;
    dasleg(plegd, nang * jdia - 1, R.xd, R.ipot, kz);
    if (R.idia == 2) {
        const int jfirst = R.zembed ? (kk + R.ipar1) % 2 : (kk + jay_ipar) % 2;
        for (int i = 1; i <= R.ipot; ++i) {
            int index = jfirst;
            for (int ll = 0; ll <= nang - 1; ++ll) {
                plegd[(i - 1) + (size_t)R.ipot * ll] = plegd[(i - 1) + (size_t)R.ipot * index];
                index += 2;
            }
        }
    }
    // d(:, ipt..ipt+ipot-1) = temp(:, jpt..jpt+nang-1) plegd^T, per radial function
    d.assign((size_t)ne * nrad * R.ipot, 0.0);
    for (int mn = 0; mn < nrad; ++mn)
        for (int i = 0; i < R.ipot; ++i)
            for (int l = 0; l < nang; ++l) {
                const double p = plegd[(size_t)i + (size_t)R.ipot * l];
                const double *src = &temp[(size_t)ne * ((size_t)mn * nang + l)];
                double *dst = &d[(size_t)ne * ((size_t)mn * R.ipot + i)];
                for (int ie = 0; ie < ne; ++ie) dst[ie] += src[ie] * p;
            }
    kbeg = kneed;
}

// trans :1648-1776 (NCPUS = 1): t += x1 dipol(p) dc1(:, p) dc2(:, p)^T over the points
void trans(Run &R, std::vector<double> &t, const std::vector<double> &dc1, const std::vector<double> &dc2, int k1,
           int k2, double xfac, int nu, int ipar) {
    const int j1 = R.jk1 - R.kmin1, j2 = R.jk2 - R.kmin2, kk1 = k1 - R.kmin1, kk2 = k2 - R.kmin2;
    double x1 = threej(j1, 1, j2, kk1, nu, -kk2, R.binom, R.nbin) * xfac;
    if (kk1 % 2 != 0) x1 = -x1;
    int i0 = 1;
    if (std::abs(nu) == 1 && ipar == 0) i0 = 0;
    size_t i = 0, id = 0;
    int n0 = R.npnt2;
    const int ne1 = R.neval1, ne2 = R.neval2;
    for (int nn1 = 1; nn1 <= R.npnt1; ++nn1) {
        if (R.idia == -2) n0 = nn1 - i0;
        const int niter = n0 * R.ipot;
        for (int n1 = 1; n1 <= niter; ++n1) {
            const size_t ii = i + n1, idd = id + n1;
            if (idd > R.dipol.size() || ne1 * ii > dc1.size() || ne2 * ii > dc2.size()) dfail(DVR3D_ERR_ARG);
            const double x3 = x1 * R.dipol[idd - 1];
            const double *a = &dc1[(size_t)ne1 * (ii - 1)], *b = &dc2[(size_t)ne2 * (ii - 1)];
            for (int q = 0; q < ne2; ++q) {
                const double s = x3 * b[q];
                for (int p = 0; p < ne1; ++p) t[(size_t)p + (size_t)ne1 * q] += a[p] * s;
            }
        }
        i += niter;
        id += niter;
        if (std::abs(nu) == i0 && R.idia == -2) id += R.npot;
    }
}

}  // namespace

extern "C" int oracle_dipole3(const char *deck_text, const char *ket_path, const char *bra_path, dvr3d_dipd_fn dipd,
                              dvr3d_dipsa_fn dipsa, void *user, const char *tra_path, dvr3d_dipole_result *res,
                              char *out, size_t outcap, size_t *outlen) {
    if (!deck_text || !ket_path || !bra_path || !res || (!dipd == !dipsa)) return DVR3D_ERR_ARG;
    try {
        Run R;
        R.dk = parse_dip_deck(deck_text);
        if (R.dk.ires != 0) dfail(DVR3D_ERR_UNSUPPORTED);
        SeqFile ket(ket_path), bra(bra_path);
        R.ket = &ket;
        R.bra = &bra;
        // ---- insize :198-620
        R.h1 = read_header(ket);
        R.h2 = read_header(bra);
        const Header &a = R.h1, &b = R.h2;
        if (a.idia != b.idia) dfail(DVR3D_ERR_ARG);
        R.idia = a.idia;
        R.jrot1 = a.jrot;
        R.jrot2 = b.jrot;
        R.ipar1 = a.ipar;
        R.ipar2 = b.ipar;
        R.kmin1 = a.kmin;
        R.kmin2 = b.kmin;
        R.znco1 = a.znco;
        R.znco2 = b.znco;
        if (R.jrot1 == 0 || R.jrot2 == 0) {
            R.zembed = a.zemb;
            if (R.jrot1 == 0) R.zembed = b.zemb;
            if (R.jrot1 == 0 && R.jrot2 == 0) dfail(DVR3D_ERR_ARG);  // j = 0 -> 0 not allowed
        } else if (R.idia > -2) {
            if (a.zemb != b.zemb) dfail(DVR3D_ERR_ARG);
            R.zembed = a.zemb;
        }
        if (R.idia > -2) {
            if (R.zembed) {
                if (R.ipar1 != R.ipar2 && R.idia == 2) dfail(DVR3D_ERR_ARG);
            } else if (R.ipar1 == R.ipar2 && R.idia == 2) {
                dfail(DVR3D_ERR_ARG);
            }
            R.zbisc = false;
        } else {
            R.zbisc = true;
            R.zembed = true;
            if (R.jrot1 == R.jrot2) {
                if (R.ipar1 != R.ipar2) dfail(DVR3D_ERR_ARG);
            } else if (R.ipar1 == R.ipar2) {
                dfail(DVR3D_ERR_ARG);
            }
        }
        if (a.zmor1 != b.zmor1 || a.zmor2 != b.zmor2) dfail(DVR3D_ERR_ARG);
        if (a.nmax1 != b.nmax1 || a.nmax2 != b.nmax2) dfail(DVR3D_ERR_ARG);
        R.npnt1 = a.nmax1;
        R.npnt2 = a.nmax2;
        const double toler = 1.0e-3;
        if (std::fabs(b.g1 - a.g1) > toler || std::fabs(b.g2 - a.g2) > toler) dfail(DVR3D_ERR_ARG);
        for (int i = 0; i < 3; ++i)
            if (std::fabs(b.xm[i] - a.xm[i]) > toler) dfail(DVR3D_ERR_ARG);
        R.D = Dipole{dipd, dipsa, user, a.g1, b.g2, false, false};
        std::vector<double> m2(6), m1(6);
        bra.getrow(m2.data(), 6);
        ket.getrow(m1.data(), 6);
        for (int i = 0; i < 6; ++i)
            if (std::fabs(m1[i] - m2[i]) > toler) dfail(DVR3D_ERR_ARG);
        if (R.znco1 && !R.znco2) {
            if (std::abs(R.jrot1) > 1) dfail(DVR3D_ERR_ARG);
            R.kmin1 = 0;
        }
        if (R.znco2 && !R.znco1) {
            if (std::abs(R.jrot2) > 1) dfail(DVR3D_ERR_ARG);
            R.kmin2 = 0;
        }
        // both files without Coriolis coupling: the reference's branch (:1067-1100) reads both
        // vector sets from the bra stream; not restated
        if (R.znco1 && R.znco2) dfail(DVR3D_ERR_UNSUPPORTED);
        if (R.jrot1 == 0) R.kmin1 = 1;
        R.jk1 = R.jrot1 + R.kmin1;
        if (R.jrot2 == 0) R.kmin2 = 1;
        R.jk2 = R.jrot2 + R.kmin2;
        R.mblock = R.jk1 + R.jk2 + std::min(R.jk1, R.jk2) - 2;
        R.nblock = std::min(R.dk.nblock, R.mblock);
        if (R.idia > -2) {
            R.nrade = R.npnt1 * R.npnt2;
            R.nrado = R.nrade;
            R.mbass1 = R.nrade * R.jk1 * a.lmax;
            R.mbass2 = R.nrade * R.jk2 * b.lmax;
        } else {
            R.nrade = R.npnt1 * (R.npnt1 + 1) / 2;
            R.nrado = R.npnt1 * (R.npnt1 - 1) / 2;
            auto mb = [&](int jk, int ipar, int lmax) {
                const int jt = jk / 2;
                int m = (R.nrade + R.nrado) * jt;
                if (2 * jt != jk) m += ipar == 0 ? R.nrade : R.nrado;
                return m * lmax;
            };
            R.mbass1 = mb(R.jk1, R.ipar1, a.lmax);
            R.mbass2 = mb(R.jk2, R.ipar2, b.lmax);
        }
        R.npot = R.dk.npot;
        R.ibase1 = R.dk.ibase1;
        R.ibase2 = R.dk.ibase2;
        int neval1 = a.neval, neval2 = b.neval;
        if (R.ibase1 <= 0 || R.ibase1 > neval1) R.ibase1 = 1;
        if (R.ibase2 <= 0 || R.ibase2 > neval2) R.ibase2 = 1;
        const int itot = R.jrot1 + R.jrot2 + 1 + R.kmin1 + R.kmin2;
        if (itot % 2 != 0 || std::abs(R.jrot1 - R.jrot2) > 1) dfail(DVR3D_ERR_ARG);  // selection rules
        R.neval1 = R.dk.nv1 > 0 ? std::min(R.dk.nv1, neval1 - R.ibase1 + 1) : neval1 - R.ibase1 + 1;
        R.neval2 = R.dk.nv2 > 0 ? std::min(R.dk.nv2, neval2 - R.ibase2 + 1) : neval2 - R.ibase2 + 1;
        R.nbin = R.jrot1 + R.jrot2 + 3;
        if (R.npot % 2 != 0) ++R.npot;
        if (R.npot < 2) dfail(DVR3D_ERR_DECK);
        R.nn2 = R.npot / 2;
        R.ipot = R.idia < 2 ? R.npot : R.npot / 2;
        R.D.zembed = R.zembed;
        R.D.zbisc = R.zbisc;
        // ---- main / genind
        R.nbass1 = genind(ket, R.mbass1, R.jk1);
        R.nbass2 = genind(bra, R.mbass2, R.jk2);
        // ---- dmain :708-1116
        R.binom = setfac(R.nbin);
        const int ne1 = R.neval1, ne2 = R.neval2;
        std::vector<double> tz((size_t)ne1 * ne2, 0.0), tx((size_t)ne1 * ne2, 0.0);
        R.r1.assign(R.npnt1, 0.0);
        R.r2.assign(R.npnt2, 0.0);
        bra.getrow(R.r1.data(), R.npnt1);
        if (R.idia > -2) bra.getrow(R.r2.data(), R.npnt2);
        if (R.jk2 <= 1) {
            for (int i = 0; i < 3; ++i) bra.skip();
            if (R.idia == -2) {
                bra.skip();
                bra.skip();
            }
        }
        ket.skip();
        if (R.idia > -2) ket.skip();
        if (R.jk1 <= 1) {
            for (int i = 0; i < 3; ++i) ket.skip();
            if (R.idia == -2) {
                ket.skip();
                ket.skip();
            }
        }
        std::vector<double> e1(ne1), e2(ne2);
        ket.skip();
        ket.getrow(e1.data(), ne1, R.ibase1 - 1);
        bra.skip();
        bra.getrow(e2.data(), ne2, R.ibase2 - 1);
        int kbeg1 = 0, kbeg2 = 0, iblock = 0, jblock = 0;
        const int kblock = R.nblock;
        std::vector<double> dc1, dc2, dlower, dmiddle, dupper;
        std::string txt;
        char ln[256];
        bool stop = false;
        // nu = 0
        int nu = 0;
        lagpt(R, nu);
        {
            int ks1 = 1, ip = R.ipar1;
            if (R.kmin1 > R.kmin2) {
                ks1 = 2;
                ip = 1 - ip;
            }
            int ipar11 = R.ipar1, ipar22 = R.ipar2;
            if (R.idia == -2) {
                if (R.kmin1 == 0) ipar11 = R.ipar1 + 1;
                if (R.kmin2 == 0) ipar22 = R.ipar2 + 1;
            }
            for (int k1 = ks1; k1 <= R.jk1 && !stop; ++k1) {
                const int k2 = k1 - R.kmin1 + R.kmin2;
                if (k2 > R.jk2) continue;
                ++jblock;
                if (jblock > iblock) {
                    ++iblock;
                    if (R.nbass1[k1 - 1] == 0 || R.nbass2[k2 - 1] == 0) {
                        std::snprintf(ln, sizeof(ln), "\n     Block%4d k1 =%3d to k2 =%3d skipped\n", iblock,
                                      k1 - R.kmin1, k2 - R.kmin2);
                        txt += ln;
                    } else {
                        const int kk = k1 - R.kmin1;
                        dsrd(R, dc1, ket, R.mbass1, R.nbass1[k1 - 1], ne1, k1, kbeg1, R.jk1, ip, R.ibase1, kk, nu,
                             R.ipar1);
                        dsrd(R, dc2, bra, R.mbass2, R.nbass2[k2 - 1], ne2, k2, kbeg2, R.jk2, 1 - ip, R.ibase2, kk, nu,
                             R.ipar2);
                        double xfac = 1.0;
                        if (R.idia == -2 && ((kk + ipar11) / 2 + (kk + ipar22) / 2) % 2 != 0) xfac = -xfac;
                        trans(R, tz, dc1, dc2, k1, k2, xfac, nu, 1);
                        std::snprintf(ln, sizeof(ln), "\n     Block%4d k1 =%3d to k2 =%3d completed\n", iblock,
                                      k1 - R.kmin1, k2 - R.kmin2);
                        txt += ln;
                        if (iblock >= kblock) stop = true;
                    }
                }
                ip = 1 - ip;
            }
            // nu = +/-1
            if (!stop) {
                nu = 1;
                lagpt(R, nu);
                ip = R.ipar1;
                for (int k1 = 1; k1 <= R.jk1 && !stop; ++k1) {
                    const int kk1 = k1 - R.kmin1;
                    if (R.nbass1[k1 - 1] != 0) {
                        dsrd(R, dc1, ket, R.mbass1, R.nbass1[k1 - 1], ne1, k1, kbeg1, R.jk1, ip, R.ibase1, kk1, nu,
                             R.ipar1);
                        if (k1 == 1) {  // the bra blocks k-1, k, k+1 kept in memory (:951-1003)
                            auto rd = [&](std::vector<double> &dst, int kneed, int ipx, int kk) {
                                dsrd(R, dst, bra, R.mbass2, R.nbass2[kneed - 1], ne2, kneed, kbeg2, R.jk2, ipx, R.ibase2,
                                     kk, 1, R.ipar2);
                            };
                            if (R.kmin1 == 0) {
                                if (R.kmin2 == R.kmin1) {
                                    rd(dmiddle, 1, 1 - ip, 1);
                                    if (R.jk2 != 1) rd(dupper, 2, ip, 2);
                                } else {
                                    rd(dlower, 1, ip, 0);
                                    rd(dmiddle, 2, 1 - ip, 1);
                                    if (R.jk2 != 1) rd(dupper, 3, ip, 2);
                                }
                            } else {
                                if (R.kmin2 == R.kmin1) {
                                    rd(dmiddle, 1, 1 - ip, 0);
                                    if (R.jk2 != 1) rd(dupper, 2, ip, 1);
                                } else {
                                    rd(dupper, 1, ip, 1);
                                }
                            }
                        }
                        int ipar11 = R.ipar1, ipar22 = R.ipar2;
                        if (R.idia == -2) {
                            if (R.kmin1 == 0) ipar11 = R.ipar1 + 1;
                            if (R.kmin2 == 0) ipar22 = R.ipar2 + 1;
                        }
                        if (R.jk2 > 1) {
                            nu = 1;
                            const int kk2 = kk1 + nu, k2 = kk2 + R.kmin2;
                            if (k2 <= R.jk2) {
                                ++jblock;
                                if (jblock > iblock) {
                                    ++iblock;
                                    if (R.nbass2[k2 - 1] == 0) {
                                        std::snprintf(ln, sizeof(ln), "\n     Block%4d k1 =%3d to k2 =%3d skipped\n",
                                                      iblock, k1 - R.kmin1, k2 - R.kmin2);
                                        txt += ln;
                                    } else {
                                        double xfac = -1.0 / std::sqrt(2.0);
                                        if (kk1 == 0) xfac = -1.0;
                                        if (R.idia == -2 && ((kk1 + ipar11) / 2 + (kk2 + ipar22) / 2) % 2 != 0) xfac = -xfac;
                                        if (!R.zembed && R.idia < 0) xfac = -xfac;
                                        trans(R, tx, dc1, dupper, k1, k2, xfac, nu, ip);
                                        std::snprintf(ln, sizeof(ln), "\n     Block%4d k1 =%3d to k2 =%3d completed\n",
                                                      iblock, k1 - R.kmin1, k2 - R.kmin2);
                                        txt += ln;
                                        if (iblock >= kblock) stop = true;
                                    }
                                }
                            }
                        }
                        if (!stop) {
                            nu = -1;
                            const int kk2 = kk1 + nu, k2 = kk2 + R.kmin2;
                            if (k2 >= 1) {
                                ++jblock;
                                if (jblock > iblock) {
                                    ++iblock;
                                    if (R.nbass2[k2 - 1] == 0) {
                                        std::snprintf(ln, sizeof(ln), "\n     Block%4d k1 =%3d to k2 =%3d skipped\n",
                                                      iblock, k1 - R.kmin1, k2 - R.kmin2);
                                        txt += ln;
                                    } else {
                                        double xfac = 1.0 / std::sqrt(2.0);
                                        if (kk2 == 0) xfac = 1.0;
                                        if (R.idia == -2 && ((kk1 + ipar11) / 2 + (kk2 + ipar22) / 2) % 2 != 0) xfac = -xfac;
                                        if (!R.zembed && R.idia < 0) xfac = -xfac;
                                        trans(R, tx, dc1, dlower, k1, k2, xfac, nu, ip);
                                        std::snprintf(ln, sizeof(ln), "\n     Block%4d k1 =%3d to k2 =%3d completed\n",
                                                      iblock, k1 - R.kmin1, k2 - R.kmin2);
                                        txt += ln;
                                        if (iblock >= kblock && k1 < R.jk1) stop = true;
                                    }
                                }
                            }
                        }
                    }
                    if (stop) break;
                    // :1005-1017
                    ip = 1 - ip;
                    dlower = dmiddle;
                    dmiddle = dupper;
                    if (kbeg2 != R.jk2) {
                        const int kk2 = kbeg2 + 1 - R.kmin2;
                        dsrd(R, dupper, bra, R.mbass2, R.nbass2[kbeg2], ne2, kbeg2 + 1, kbeg2, R.jk2, ip, R.ibase2, kk2,
                             nu, R.ipar2);
                    }
                }
            }
        }
        // ---- spect :1825-1954
        const double autocm = 2.19474624e+05, autode = 2.5417662, detosec = 3.136186e-07;
        const int j1 = R.jk1 - R.kmin1, j2 = R.jk2 - R.kmin2;
        std::string s;
        std::snprintf(ln, sizeof(ln), "\n     %s\n", R.dk.title.c_str());
        s += ln;
        std::snprintf(ln, sizeof(ln), "\n     j1=%4d  kmin1=%4d  j2=%4d  kmin2=%4d  idia=%4d  ipar1=%4d  ipar2=%4d\n\n",
                      j1, R.kmin1, j2, R.kmin2, R.idia, R.ipar1, R.ipar2);
        s += ln;
        if (R.dk.have_ezero) {
            std::snprintf(ln, sizeof(ln), "     ground zero =%s cm-1\n", fmt_fd(R.dk.ezero, 16, 8, 'E').c_str());
            s += ln;
        }
        s += "\n ie1 ie2   ket energy   bra energy    frequency  z transition    x transition       dipole       "
             "s(f-i)      a-coefficient\n\n";
        const double xf = std::sqrt((double)((2 * j1 + 1) * (2 * j2 + 1)));
        std::vector<double> sint((size_t)ne1 * ne2), xe2(ne2);
        for (int ie1 = 1; ie1 <= ne1; ++ie1) {
            const double xe1 = e1[ie1 - 1] * autocm - R.dk.ezero;
            for (int ie2 = 1; ie2 <= ne2; ++ie2) {
                if (ie1 == 1) xe2[ie2 - 1] = e2[ie2 - 1] * autocm - R.dk.ezero;
                const double dd = xe2[ie2 - 1] - xe1;
                const double dd3 = std::fabs(dd * dd * dd);
                const size_t q = (size_t)(ie1 - 1) + (size_t)ne1 * (ie2 - 1);
                const double sx = (tz[q] + tx[q]) * (tz[q] + tx[q]);
                sint[q] = sx * xf * xf;
                const double tzd = tz[q] * autode * xf;
                double txd = tx[q] * autode * xf;
                if (!R.zbisc && R.zembed) txd = -txd;
                const double t = std::fabs(tzd + txd), sxd = t * t;
                double av = 0.0;
                if (dd > 0.0) av = sxd * dd3 * detosec / (double)(2 * j2 + 1);
                if (dd < 0.0) av = sxd * dd3 * detosec / (double)(2 * j1 + 1);
                if (R.dk.zpmin && std::max(ie1, ie2) > 10) continue;
                std::snprintf(ln, sizeof(ln), "%4d%4d   %14.6f   %14.6f   %14.6f  %s  %s  %s  %s  %s\n", ie1, ie2, xe1,
                              xe2[ie2 - 1], dd, fmt_es(tzd, 15, 8).c_str(), fmt_es(txd, 15, 8).c_str(),
                              fmt_es(t, 15, 8).c_str(), fmt_es(sxd, 15, 8).c_str(), fmt_es(av, 15, 8).c_str());
                s += ln;
            }
        }
        // ---- outpt :1956-2003
        if (R.dk.ztra && tra_path && tra_path[0]) {
            FILE *fp = std::fopen(tra_path, R.dk.zstart ? "wb" : "ab");
            if (!fp) dfail(DVR3D_ERR_ARG);
            auto put = [&](const void *p, size_t n) {
                const int32_t m = (int32_t)n;
                std::fwrite(&m, 4, 1, fp);
                std::fwrite(p, 1, n, fp);
                std::fwrite(&m, 4, 1, fp);
            };
            unsigned char h[56];
            const int hi[9] = {j1, j2, R.kmin1, R.kmin2, ne1, ne2, R.idia, R.ipar1, R.ipar2};
            std::memcpy(h, hi, 36);
            std::memcpy(h + 36, &R.dk.ezero, 8);
            const int32_t ze = R.zembed ? 1 : 0;
            std::memcpy(h + 44, &ze, 4);
            const int hb[2] = {R.ibase1, R.ibase2};
            std::memcpy(h + 48, hb, 8);
            put(h, 56);
            put(e1.data(), 8 * (size_t)ne1);
            put(e2.data(), 8 * (size_t)ne2);
            for (int ie2 = 0; ie2 < ne2; ++ie2) put(&sint[(size_t)ne1 * ie2], 8 * (size_t)ne1);
            std::fclose(fp);
        }
        // ---- results
        if (res->cap1 < ne1 || res->cap2 < ne2) dfail(DVR3D_ERR_BUFFER);
        res->neval1 = ne1;
        res->neval2 = ne2;
        res->j1 = j1;
        res->j2 = j2;
        res->kmin1 = R.kmin1;
        res->kmin2 = R.kmin2;
        res->nblocks = iblock;
        auto put2 = [&](double *dst, const std::vector<double> &src) {
            if (!dst) return;
            for (int q = 0; q < ne2; ++q)
                for (int p = 0; p < ne1; ++p) dst[(size_t)p + (size_t)res->cap1 * q] = src[(size_t)p + (size_t)ne1 * q];
        };
        put2(res->tz, tz);
        put2(res->tx, tx);
        put2(res->sint, sint);
        if (res->e1) std::memcpy(res->e1, e1.data(), 8 * (size_t)ne1);
        if (res->e2) std::memcpy(res->e2, e2.data(), 8 * (size_t)ne2);
        std::string all = txt + s;
        if (outlen) *outlen = all.size();
        if (out && outcap) {
            const size_t n = std::min(all.size(), outcap - 1);
            std::memcpy(out, all.data(), n);
            out[n] = 0;
        }
        return DVR3D_OK;
    } catch (DFail &f) {
        return f.code;
    }
}

// The angular quadrature of lagpt (jacobi with alf = bta = 0): the nn2 largest points, their
// weights, and the computed and exact half sums.
extern "C" int oracle_dipole_quadrature(int npot, double *x, double *w, double *csa, double *tsa) {
    if (npot < 2 || npot % 2 || !x || !w || !csa || !tsa) return DVR3D_ERR_ARG;
    try {
        std::vector<double> b(npot + 1, 0.0), c(npot + 1, 0.0), xx(npot + 1, 0.0), a(npot + 1, 0.0);
        for (int i = 2; i <= npot; ++i) {
            const double xi = (double)i;
            c[i] = 4.0 * (xi - 1.0) * (xi - 1.0) * (xi - 1.0) * (xi - 1.0) /
                   ((2.0 * xi - 1.0) * (2.0 * xi - 2.0) * (2.0 * xi - 2.0) * (2.0 * xi - 3.0));
        }
        djacobi(npot, xx, a, 0.0, 0.0, b, c, *csa, *tsa);
        for (int i = 1; i <= npot / 2; ++i) {
            x[i - 1] = xx[i];
            w[i - 1] = a[i];
        }
        return DVR3D_OK;
    } catch (DFail &f) {
        return f.code;
    }
}

// threej of the reference on its binomial table (for known-answer tests)
extern "C" double oracle_threej(int j1, int j2, int j3, int m1, int m2, int m3) {
    const int nbin = j1 + j2 + j3 + 3;
    try {
        return threej(j1, j2, j3, m1, m2, m3, setfac(nbin), nbin);
    } catch (DFail &) {
        return std::nan("");
    }
}
