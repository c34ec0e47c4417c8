// rotlev.cu -- the second variational step for J > 0 in symmetrised Radau coordinates with the
// bisector embedding: the reference's ROTLEV3B (source/rotlev3b_segmented.f90).
//
// Input: the wavefunction file (unit IVEC, fort.26) that the first step wrote for the k blocks
// of one J (dvr3d_b200_run_deck_wave with ZROT, ZTRAN), and ROTLEV3B's job deck. The rotational
// Hamiltonian in the basis of the lowest vibrational functions of every k block has
//   * on its diagonal the vibrational levels of each block (select :306-510);
//   * Coriolis blocks between k and k+1 and between k and k+2 (solrt :1339-1620): an angular
//     matrix in the DVR of the two blocks (angin1 :719-814, angin2 :816-873, from a Gauss-
//     associated Legendre quadrature in the FBR), combined with the symmetrised radial r^-2
//     matrix elements (radint / mkrad :665-717) and the two blocks' first-step vectors
//     (solofd :1682-1729).
// solofd's sum over radial pairs of radmat(ir) (A C2_ir2)^T C1_ir1 runs here as two DMMA GEMMs
// per block pair: W = A C2 over all radial blocks and vectors at once, then offdg = W''^T C1''
// with W'' and C1'' the radial blocks each pair uses, gathered (and W'' scaled) by one kernel.
// The Hamiltonian is assembled on the device and its lowest levels come from the dense FP64
// eigensolver (dgrot's dsyev path :1752-1757; its iterative path gives the same levels).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iterator>
#include <string>
#include <vector>

#include "../../include/dvr3d_b200.h"
#include "common.cuh"
#include "gemm64.cuh"
#include "pipeline.cuh"
#include "rotlev.cuh"
#include "wavefile.cuh"

#define CK(x)                                          \
    do {                                               \
        cudaError_t e_ = (x);                          \
        if (e_ != cudaSuccess) throw CudaFail{e_, #x}; \
    } while (0)

namespace dvr3d {

namespace {

[[noreturn]] void bad(int code, const std::string &m) { throw HostError{code, m}; }

// One k block of the file (ccmain :972-976, testiv :3446-3448, transr :3622-3641).
struct KBlock {
    int k = 0, maxleg = 0, nang = 0, lincr = 0, iang = 0, ibass = 0, meval = 0;
    std::vector<double> pleg;  // pleg(j, i) * walf(i), (maxleg + 1) x nang
    std::vector<int> iv;       // kept 2D states per angle
    std::vector<double> ev;    // levels (Eh)
    size_t vec0 = 0;           // record index of the first vector
    size_t xalf_rec = 0;       // record index of the block's angular points
};

// ROTLEV3B's cards after the namelist (insize :157-161): nvib, neval, kmin, ibass, neval2,
// npnt (12i5), the title, and the optional EZERO card (vrmain :593-596).
struct RotDeck {
    int nvib = 0, neval = 0, kmin = 0, ibass = 0, neval2 = 0, npnt = 0;
    std::string title;
    double ezero = 0.0;
};

int field_i5(const std::string &ln, int i) {
    if ((size_t)(5 * i) >= ln.size()) return 0;
    const std::string s = ln.substr(5 * i, 5);
    try {
        size_t used = 0;
        const std::string t = s.substr(s.find_first_not_of(' ') == std::string::npos ? s.size() : s.find_first_not_of(' '));
        if (t.empty()) return 0;
        return std::stoi(t, &used);
    } catch (...) {
        bad(DVR3D_ERR_DECK, "ROTLEV3B card: not an integer in columns " + std::to_string(5 * i + 1));
    }
}

RotDeck parse_rot_deck(const char *text) {
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
    // the namelist: from the line with '&' up to the line holding its closing '/'
    size_t i = 0;
    while (i < lines.size() && lines[i].find('&') == std::string::npos) ++i;
    if (i == lines.size()) bad(DVR3D_ERR_DECK, "ROTLEV3B deck: no namelist PRT");
    while (i < lines.size() && lines[i].find('/') == std::string::npos) ++i;
    ++i;
    if (i >= lines.size()) bad(DVR3D_ERR_DECK, "ROTLEV3B deck: no card after the namelist");
    RotDeck d;
    d.nvib = field_i5(lines[i], 0);
    d.neval = field_i5(lines[i], 1);
    d.kmin = field_i5(lines[i], 2);
    d.ibass = field_i5(lines[i], 3);
    d.neval2 = field_i5(lines[i], 4);
    d.npnt = field_i5(lines[i], 5);
    if (i + 1 < lines.size()) d.title = lines[i + 1].substr(0, 72);
    if (i + 2 < lines.size()) {
        const std::string e = lines[i + 2].substr(0, std::min<size_t>(20, lines[i + 2].size()));
        if (e.find_first_not_of(' ') != std::string::npos) {
            std::string t = e;
            for (auto &ch : t)
                if (ch == 'd' || ch == 'D') ch = 'e';
            try {
                d.ezero = std::stod(t);
            } catch (...) {
                bad(DVR3D_ERR_DECK, "ROTLEV3B deck: EZERO card is not a number");
            }
        }
    }
    return d;
}

// Gauss-associated Legendre rule of ROTLEV3B's jacobi (:941-1007): zeros of the Jacobi
// polynomial P_n^(k,k) found by a downward sign scan from x = 1 in steps of 1e-6, refined by
// Newton (10 steps at most, |dx| <= 1e-12) with the derivative of the last evaluation; weights
// from the recurrence constant. Returned over the full range, ascending (angin1 :760-764).
void rot_quadrature(int n, int k, std::vector<double> &x, std::vector<double> &w, double &cs, double &ts) {
    const double a = k, b = k;
    std::vector<double> c(n + 1, 0.0);
    for (int i = 2; i <= n; ++i) {
        const double xi = (float)i;
        c[i] = 4.0 * (xi - 1.0) * (a + xi - 1.0) * (b + xi - 1.0) * (a + b + xi - 1.0) /
               ((a + b + 2.0 * xi - 1.0) * (a + b + 2.0 * xi - 2.0) * (a + b + 2.0 * xi - 2.0) * (a + b + 2.0 * xi - 3.0));
    }
    ts = std::pow(2.0, k + k + 1) / (double)(k + 1);
    for (int i = 1; i <= k; ++i) ts = ts * (double)i / (double)(k + i + 1);
    double cc = ts;
    for (int i = 2; i <= n; ++i) cc *= c[i];
    auto recur = [&](double xx, double &p, double &dp, double &p1) {
        double pa = 1.0, pb = xx + (a - b) / (a + b + 2.0), da = 0.0, db = 1.0;
        for (int j = 2; j <= n; ++j) {
            const double q = xx * pb - c[j] * pa;
            const double dq = xx * db + pb - c[j] * da;
            pa = pb;
            pb = q;
            da = db;
            db = dq;
        }
        p = pb;
        dp = db;
        p1 = pa;
    };
    const int n2 = (n + 1) / 2;
    std::vector<double> xt;
    const double xstep = 1.0e-6;
    double pm1 = 1.0, xx = 1.0;
    for (;;) {
        double p, dp, p1;
        recur(xx, p, dp, p1);
        if (pm1 * p < 0.0) {
            pm1 = -pm1;
            xt.push_back(xx - 0.5 * xstep);
        }
        if ((int)xt.size() == n2) break;
        xx -= xstep;
        if (!(xx > -1.5 * xstep)) bad(DVR3D_ERR_QUADRATURE, "ROTLEV3B quadrature: wrong number of zeros found");
    }
    std::vector<double> xh(n2), wh(n2);
    cs = 0.0;
    for (int i = 0; i < n2; ++i) {
        double z = xt[i], p = 0, dp = 1, p1 = 0;
        for (int it = 0; it < 10; ++it) {
            recur(z, p, dp, p1);
            const double dlt = p / dp;
            z -= dlt;
            if (std::fabs(dlt) <= 1.0e-12) break;
        }
        xh[i] = z;
        wh[i] = cc / (dp * p1);
        cs += wh[i] + wh[i];
    }
    if (2 * n2 != n) cs -= wh[n2 - 1];
    x.assign(n, 0.0);
    w.assign(n, 0.0);
    for (int i = 0; i < n2; ++i) {
        x[n - 1 - i] = xh[i];
        w[n - 1 - i] = wh[i];
        x[i] = -xh[i];
        w[i] = wh[i];
    }
}

// ROTLEV3B's asleg (:1051-1157) for m < 90: polynomial parts of the normalised associated
// Legendre functions P_l^m, l = m .. m + lmax, at the points x -> p((lmax+1) x npt).
std::vector<double> rot_asleg(const std::vector<double> &x, int lmax, int m) {
    const int npt = (int)x.size();
    if (m < 0 || m >= 90) bad(DVR3D_ERR_UNSUPPORTED, "ROTLEV3B angular functions for k >= 90");
    std::vector<double> p((size_t)(lmax + 1) * npt, 0.0);
    for (int i = 0; i < npt; ++i) {
        double pmm = 1.0, f = 1.0;
        for (int j = 1; j <= m; ++j) {
            pmm = -pmm * f;
            f += 2.0;
        }
        double *col = &p[(size_t)i * (lmax + 1)];
        col[0] = pmm;
        double pmmp1 = x[i] * (m + m + 1) * pmm;
        if (lmax >= 1) col[1] = pmmp1;
        int ll = 1;
        for (int l = 2 + m; l <= lmax + m; ++l) {
            const double pll = (x[i] * (double)(l + l - 1) * pmmp1 - (double)(l + m - 1) * pmm) / (double)(l - m);
            pmm = pmmp1;
            pmmp1 = pll;
            col[++ll] = pll;
        }
    }
    for (int j = m, jj = 0; j <= lmax + m; ++j, ++jj) {
        double f = 1.0;
        for (int i = j - m + 1; i <= j + m; ++i) f *= std::sqrt((double)i);
        const double nrm = std::sqrt(((double)j + (double)j + 1.0) / 2) / f;
        for (int i = 0; i < npt; ++i) p[(size_t)i * (lmax + 1) + jj] *= nrm;
    }
    return p;
}

// Angular Coriolis matrix between the kept angles of two k blocks (angin1 / angin2): the FBR
// integral over the quadrature, transformed to the two DVRs by the blocks' own pleg * walf.
// step 1: blocks k1 and k1+1, weight (1 + x); step 2: k1 and k1+2, weight (1 + x)^2.
std::vector<double> angular_block(int step, int k1, const KBlock &b1, const KBlock &b2, int npnt,
                                  double angfac) {
    std::vector<double> x, w;
    double cs = 0, ts = 0;
    rot_quadrature(npnt, k1, x, w, cs, ts);
    if (std::fabs((cs - ts) / ts) > 1.0e-8) bad(DVR3D_ERR_QUADRATURE, "ROTLEV3B points & weights in error");
    const int n1 = b1.nang, n2 = b2.nang;
    const std::vector<double> pa = rot_asleg(x, n1 - 1, k1);
    const std::vector<double> pb = rot_asleg(x, n2 - 1, k1 + step);
    std::vector<double> fbr((size_t)n1 * n2, 0.0);  // fbr(j, k), column-major n1 x n2
    for (int i = 0; i < npnt; ++i) {
        const double t = step == 1 ? w[i] * (1.0 + x[i]) : w[i] * ((1.0 + x[i]) * (1.0 + x[i]));
        for (int j = 0; j < n1; ++j) {
            const double f = t * pa[(size_t)i * n1 + j];
            for (int k = 0; k < n2; ++k) fbr[(size_t)k * n1 + j] += f * pb[(size_t)i * n2 + k];
        }
    }
    // the file's transforms: pleg(j, i) with leading dimension maxleg + 1
    const int ld1 = b1.maxleg + 1, ld2 = b2.maxleg + 1;
    auto P1 = [&](int j, int i) { return b1.pleg[(size_t)i * ld1 + j]; };
    auto P2 = [&](int j, int i) { return b2.pleg[(size_t)i * ld2 + j]; };
    std::vector<double> ang((size_t)b1.iang * b2.iang, 0.0);  // column-major iang1 x iang2
    const double kkp1 = (double)k1 * (k1 + 1), xkph = k1 + 0.5;
    int i1 = 0;
    for (int i = 0; i < n1; ++i) {
        if (b1.iv[i] == 0) continue;
        int i2 = 0;
        for (int ip = 0; ip < n2; ++ip) {
            if (b2.iv[ip] == 0) continue;
            double sum1 = 0.0, sum2 = 0.0;
            for (int j = 0; j < n1; ++j) {
                if (step == 1 && j > 0) {
                    const double jj = k1 + j;
                    sum1 += P1(j, i) * P2(j - 1, ip) * std::sqrt(jj * (jj + 1.0) - kkp1);
                }
                for (int jp = 0; jp < n2; ++jp) sum2 += P1(j, i) * P2(jp, ip) * fbr[(size_t)jp * n1 + j];
            }
            ang[(size_t)i2 * b1.iang + i1] = (step == 1 ? sum1 + xkph * sum2 : sum2) * angfac;
            ++i2;
        }
        ++i1;
    }
    return ang;
}

// W''[(ir, a), v] = rad[ir] * W[a + (m2[ir] + v * nrad2) * iang1];  C1''[(ir, a), v] = C1[a + m1[ir] * iang1 + v * ldc1]
__global__ void rot_gather_kernel(const double *W, int iang1, int nrad2, int nvec2, const double *C1, long long ldc1,
                                  int nvec1, const int *m1, const int *m2, const double *rad, int npair, double *Wg,
                                  double *Cg) {
    const long long K = (long long)npair * iang1;
    const long long tot = K * (long long)(nvec1 > nvec2 ? nvec1 : nvec2);
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += (long long)gridDim.x * blockDim.x) {
        const long long row = t % K;
        const int v = (int)(t / K);
        const int ir = (int)(row / iang1), a = (int)(row % iang1);
        if (v < nvec2) Wg[(size_t)v * K + row] = rad[ir] * W[a + ((long long)m2[ir] + (long long)v * nrad2) * iang1];
        if (v < nvec1) Cg[(size_t)v * K + row] = C1[a + (long long)m1[ir] * iang1 + (long long)v * ldc1];
    }
}

// H(r0 + v1, c0 + v2) = H(c0 + v2, r0 + v1) = off(v2, v1) (off: n2 x n1)
__global__ void rot_place_kernel(const double *off, int n2, int n1, double *H, long long ldh, int r0, int c0) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < (long long)n1 * n2;
         t += (long long)gridDim.x * blockDim.x) {
        const int v2 = (int)(t % n2), v1 = (int)(t / n2);
        const double x = off[t];
        H[(size_t)(c0 + v2) * ldh + (r0 + v1)] = x;
        H[(size_t)(r0 + v1) * ldh + (c0 + v2)] = x;
    }
}

__global__ void rot_diag_kernel(const double *e, int n, double *H, long long ldh) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) H[(size_t)i * ldh + i] = e[i];
}

unsigned nblocks256(long long n) { return (unsigned)std::min<long long>((n + 255) / 256, 4096); }

std::string fmt_d(double v, int w, int d) {
    // Fortran Dw.d: 0.ddddD+ee
    char buf[64];
    if (v == 0.0) {
        std::snprintf(buf, sizeof(buf), "0.%0*dD+00", d, 0);
    } else {
        int ex = (int)std::floor(std::log10(std::fabs(v))) + 1;
        double mant = std::fabs(v) / std::pow(10.0, ex);
        const double scale = std::pow(10.0, d);
        double rm = std::round(mant * scale);
        if (rm >= scale) {
            rm /= 10.0;
            ex += 1;
        }
        if (rm < scale / 10.0) {
            rm *= 10.0;
            ex -= 1;
        }
        std::snprintf(buf, sizeof(buf), "%s0.%0*.0fD%c%02d", v < 0 ? "-" : "", d, rm, ex < 0 ? '-' : '+', std::abs(ex));
    }
    std::string s(buf);
    if ((int)s.size() < w) s = std::string(w - s.size(), ' ') + s;
    return s;
}

}  // namespace

void rotlev3b_solve(dvr3d_ctx *ctx, const char *deck_text, const char *wave_path, std::vector<double> &levels,
                    std::string &table, RotInfo &info, const char *kvec_path, std::vector<double> *levels_f,
                    const char *kvec2_path) {
    const RotDeck rd = parse_rot_deck(deck_text);
    Records f(wave_path);
    // ---- header (setcon :1176-1184 as insize :155 reads it)
    const std::vector<int> h = f.ints(9);
    const int idia = h[0], ipar0 = h[1], ndvr = h[2], nmax = h[3], jrot = h[5], kmin0 = h[6], meval = h[7];
    if (idia != -2) bad(DVR3D_ERR_UNSUPPORTED, "ROTLEV3B reads Radau (IDIA = -2) wavefunction files");
    if (jrot <= 0) bad(DVR3D_ERR_ARG, "ROTLEV3B needs a J > 0 wavefunction file");
    const int kmin = rd.kmin;
    if (kmin != kmin0 && kmin0 != 2) bad(DVR3D_ERR_ARG, "ROTLEV3B: kmin differs from the first step's kmin");
    if (kmin > 2 || (kmin == 0 && kmin0 != 0))
        bad(DVR3D_ERR_UNSUPPORTED, "ROTLEV3B: kmin 0 needs a file of kmin 0; kmin 1 a file of kmin 1 or 2; kmin 2 both");
    if (kmin == 2 && !levels_f) bad(DVR3D_ERR_ARG, "ROTLEV3B with KMIN = 2 returns two sets: use the pair entry point");
    const auto flags = f.take();                             // logical flags, masses, g1, g2
    const std::vector<double> morse = f.dbls(6);             // Morse constants
    const std::vector<double> rm2 = f.dbls((size_t)nmax);    // r^-2 term (ccmain :824-833)
    const std::vector<double> rgrid = f.dbls((size_t)nmax);  // r
    if (flags.second < 56) bad(DVR3D_ERR_ARG, "wavefunction file: short flags record");
    // ---- k blocks
    const int nblk = kmin > 0 ? jrot + 1 : jrot;
    auto read_block = [&]() {
        KBlock b;
        b.xalf_rec = f.next;
        f.take();  // xalf
        const std::vector<int> hk = f.ints(4);
        b.k = hk[0];
        b.maxleg = hk[1];
        b.nang = hk[2];
        b.lincr = hk[3];
        b.pleg = f.dbls((size_t)(b.maxleg + 1) * b.nang);
        const std::vector<int> ib = f.ints(2);
        b.iang = ib[0];
        b.ibass = ib[1];
        b.iv = f.ints((size_t)b.nang);
        b.meval = f.ints(1)[0];
        b.ev = f.dbls((size_t)b.meval);
        b.vec0 = f.next;
        f.next += (size_t)b.meval;
        if (f.next > f.rec.size()) bad(DVR3D_ERR_ARG, "wavefunction file: ends inside the vectors of a k block");
        if (b.iang <= 0 || b.ibass % b.iang != 0) bad(DVR3D_ERR_ARG, "wavefunction file: inconsistent basis sizes");
        return b;
    };
    std::vector<KBlock> kb;
    while ((int)kb.size() < nblk && f.more()) kb.push_back(read_block());
    if ((int)kb.size() < nblk) bad(DVR3D_ERR_ARG, "wavefunction file holds fewer k blocks than J + 1 - kmin");
    for (int i = 0; i < nblk; ++i)
        if (kb[i].k != (kmin > 0 ? i : i + 1)) bad(DVR3D_ERR_ARG, "wavefunction file: unexpected k block order");
    // KMIN = 2: the f-type k = 1 block follows the J + 1 e-type blocks (endiv :1635-1658)
    KBlock kf1;
    if (kmin == 2) {
        if (!f.more()) bad(DVR3D_ERR_ARG, "wavefunction file: no f-type k = 1 block after the e blocks (KMIN = 2)");
        kf1 = read_block();
        if (kf1.k != 1) bad(DVR3D_ERR_ARG, "wavefunction file: the block after the e blocks is not k = 1");
    }
    // ---- basis selection (select :306-510)
    const int nvib = std::min(rd.nvib, meval);
    std::vector<int> mvib(nblk);
    int ipt = 0;
    for (int i = 0; i < nblk; ++i) {
        mvib[i] = std::min({nvib, kb[i].ibass, kb[i].meval});
        ipt += mvib[i];
    }
    int nbass = ipt;
    if (rd.ibass > 0 && rd.ibass < ipt) {  // the ibass lowest functions over all blocks
        std::vector<int> iv(nblk, 0);
        for (int n = 0; n < rd.ibass; ++n) {
            int jpt = -1;
            double e = 0.0;
            for (int j = 0; j < nblk; ++j) {
                if (iv[j] >= mvib[j]) continue;
                if (jpt < 0 || kb[j].ev[iv[j]] < e) {
                    e = kb[j].ev[iv[j]];
                    jpt = j;
                }
            }
            ++iv[jpt];
        }
        mvib = iv;
        nbass = rd.ibass;
    }
    int neval = rd.neval <= 0 ? 10 : rd.neval;
    const int neval2 = rd.neval2 <= 0 ? neval : rd.neval2;
    neval = std::min(neval, nbass);
    const int npnt = std::max(ndvr, rd.npnt);
    // ---- symmetrised radial r^-2 matrix elements (mkrad :698-717)
    auto mkrad = [&](int iq, int ip, int is) {
        std::vector<double> r;
        const double symm = 1 - 2 * ip, sign = 1 - 2 * is;
        for (int i1 = 0; i1 < nmax; ++i1)
            for (int i2 = 0; i2 < i1 + 1 - iq; ++i2) r.push_back(sign * (rm2[i2] + symm * rm2[i1]));
        return r;
    };
    const std::vector<double> radmee = mkrad(0, 0, 0), radmoo = mkrad(1, 0, 0), radmeo = mkrad(1, 1, 0),
                              radmoe = mkrad(1, 1, 1);
    cudaStream_t st = ctx->stream;
    // first-step vectors of a block, on the device (ibass x nv)
    auto upload_vectors = [&](const KBlock &b, int nv, const char *name) {
        double *d = ctx->arena.get_t<double>(name, (size_t)b.ibass * std::max(nv, 1));
        for (int v = 0; v < nv; ++v)
            CK(cudaMemcpyAsync(d + (size_t)v * b.ibass, f.vec(b.vec0 + v, (size_t)b.ibass), sizeof(double) * b.ibass,
                               cudaMemcpyHostToDevice, st));
        CK(cudaStreamSynchronize(st));
        return d;
    };
    const double jjp1 = (double)jrot * (jrot + 1);
    info.offdiag_flops = 0.0;
    // The Hamiltonian of a chain of k blocks on the device (solrt :1414-1527, loadh): each block's
    // levels on the diagonal, the Coriolis blocks of neighbours k, k+1 and k, k+2 (solofd); ip0
    // is the radial parity label of the first pair, alternating along the chain. Returns the
    // lowest nev levels, and the eigenvectors in Z (ldz) when asked.
    struct Pass {
        std::vector<int> off;
        int nb = 0;
        long long ldz = 0;
        double *Z = nullptr;
    };
    auto solve_chain = [&](const std::vector<const KBlock *> &B, const std::vector<int> &mv, int ip0, int nev,
                           bool vecs, std::vector<double> &lv, const char *tag) {
        Pass ps;
        const int nk = (int)B.size();
        ps.off.assign(nk + 1, 0);
        for (int i = 0; i < nk; ++i) ps.off[i + 1] = ps.off[i] + mv[i];
        const int nb = ps.off[nk];
        ps.nb = nb;
        const long long ldh = (nb + 7) / 8 * 8;
        double *H = ctx->arena.get_t<double>("rt_h", (size_t)ldh * nb);
        CK(cudaMemsetAsync(H, 0, sizeof(double) * ldh * nb, st));
        {
            std::vector<double> dg(nb);
            for (int i = 0; i < nk; ++i)
                for (int v = 0; v < mv[i]; ++v) dg[ps.off[i] + v] = B[i]->ev[v];
            double *dd = ctx->arena.get_t<double>("rt_dg", nb);
            CK(cudaMemcpyAsync(dd, dg.data(), sizeof(double) * nb, cudaMemcpyHostToDevice, st));
            DVR3D_COUNT_LAUNCH(1);
            rot_diag_kernel<<<nblocks256(nb), 256, 0, st>>>(dd, nb, H, ldh);
            CK(cudaGetLastError());
            CK(cudaStreamSynchronize(st));
        }
        // one Coriolis block (solofd): off (n2 x n1), placed at rows of block i, columns of block j
        auto coriolis = [&](int i, int j, const std::vector<double> &ang, const std::vector<double> &rad, int iq,
                            int iq1, int iq2) {
            const KBlock &b1 = *B[i], &b2 = *B[j];
            const int n1 = mv[i], n2 = mv[j];
            if (n1 == 0 || n2 == 0) return;
            const int nrad2 = b2.ibass / b2.iang;
            std::vector<int> m1, m2;
            int ir1 = 0, ir2 = 0;
            for (int a1 = 0; a1 < nmax; ++a1) {
                for (int a2 = 0; a2 < a1 + 1 - iq; ++a2) {
                    m1.push_back(ir1++);
                    m2.push_back(ir2++);
                }
                ir1 += iq1;
                ir2 += iq2;
            }
            const int npair = (int)m1.size();
            if (ir1 > b1.ibass / b1.iang || ir2 > nrad2 || (int)rad.size() != npair)
                bad(DVR3D_ERR_ARG, "wavefunction file: radial basis does not match the block parities");
            double *C1 = upload_vectors(b1, n1, "rt_c1");
            double *C2 = upload_vectors(b2, n2, "rt_c2");
            double *A = ctx->arena.get_t<double>("rt_ang", ang.size());
            CK(cudaMemcpyAsync(A, ang.data(), sizeof(double) * ang.size(), cudaMemcpyHostToDevice, st));
            const long long K = (long long)npair * b1.iang;
            double *W = ctx->arena.get_t<double>("rt_w", (size_t)b1.iang * nrad2 * n2);
            double *Wg = ctx->arena.get_t<double>("rt_wg", (size_t)K * n2);
            double *Cg = ctx->arena.get_t<double>("rt_cg", (size_t)K * n1);
            double *O = ctx->arena.get_t<double>("rt_off", (size_t)n1 * n2);
            int *dm1 = ctx->arena.get_t<int>("rt_m1", npair), *dm2 = ctx->arena.get_t<int>("rt_m2", npair);
            double *dr = ctx->arena.get_t<double>("rt_rad", npair);
            CK(cudaMemcpyAsync(dm1, m1.data(), sizeof(int) * npair, cudaMemcpyHostToDevice, st));
            CK(cudaMemcpyAsync(dm2, m2.data(), sizeof(int) * npair, cudaMemcpyHostToDevice, st));
            CK(cudaMemcpyAsync(dr, rad.data(), sizeof(double) * npair, cudaMemcpyHostToDevice, st));
            // W (iang1 x nrad2 n2) = A (iang1 x iang2) C2 (iang2 x nrad2 n2)
            launch_dgemm(false, false, b1.iang, nrad2 * n2, b2.iang, 1.0, A, b1.iang, C2, b2.iang, 0.0, W, b1.iang, st);
            CK(cudaGetLastError());
            DVR3D_COUNT_LAUNCH(1);
            rot_gather_kernel<<<nblocks256(K * std::max(n1, n2)), 256, 0, st>>>(W, b1.iang, nrad2, n2, C1, b1.ibass, n1,
                                                                                 dm1, dm2, dr, npair, Wg, Cg);
            CK(cudaGetLastError());
            // off (n2 x n1) = W''^T C1''
            launch_dgemm(true, false, n2, n1, (int)K, 1.0, Wg, K, Cg, K, 0.0, O, n2, st);
            CK(cudaGetLastError());
            DVR3D_COUNT_LAUNCH(1);
            rot_place_kernel<<<nblocks256((long long)n1 * n2), 256, 0, st>>>(O, n2, n1, H, ldh, ps.off[i], ps.off[j]);
            CK(cudaGetLastError());
            CK(cudaStreamSynchronize(st));
            info.offdiag_flops += 2.0 * b1.iang * b2.iang * (double)nrad2 * n2 + 2.0 * (double)K * n1 * n2;
        };
        int ip = ip0;
        for (int i = 1; i < nk; ++i) {
            const int k1 = B[i - 1]->k;
            // k and k + 1 (solrt :1468-1486)
            double angfac = std::sqrt(jjp1 - (double)k1 * (k1 + 1)) / 2.0;
            if (k1 == 0) angfac = 1.4142135623731 * angfac;
            if (mv[i - 1] * mv[i] > 0) {
                const std::vector<double> ang = angular_block(1, k1, *B[i - 1], *B[i], npnt, angfac);
                if (ip == 0) coriolis(i - 1, i, ang, radmeo, 1, 1, 0);
                else coriolis(i - 1, i, ang, radmoe, 1, 0, 1);
            }
            // k and k + 2 (:1488-1520)
            if (i + 1 < nk && mv[i - 1] * mv[i + 1] > 0) {
                double af = -std::sqrt((jjp1 - (double)(k1 + 1) * (k1 + 2)) * (jjp1 - (double)k1 * (k1 + 1))) / 16.0;
                if (k1 == 0) af = 1.4142135623731 * af;
                const std::vector<double> ang = angular_block(2, k1, *B[i - 1], *B[i + 1], npnt, af);
                if (ip == 0) coriolis(i - 1, i + 1, ang, radmee, 0, 0, 0);
                else coriolis(i - 1, i + 1, ang, radmoo, 1, 0, 0);
            }
            ip = 1 - ip;
        }
        // ---- lowest levels (dgrot)
        double *wv = ctx->arena.get_t<double>("rt_w_ev", nev);
        ps.ldz = ldh;
        ps.Z = vecs ? ctx->arena.get_t<double>(std::string("rt_z") + tag, (size_t)ps.ldz * nev) : nullptr;
        dense_lowest(ctx, H, ldh, nb, nev, vecs, wv, ps.Z, vecs ? ps.ldz : 1, "rtd_", false, nullptr);
        lv.resize(nev);
        CK(cudaMemcpyAsync(lv.data(), wv, sizeof(double) * nev, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        return ps;
    };
    // ZTRAN: the vectors back in the first step's basis, angular FBR (dstore :1917-2049)
    auto write_kvec = [&](const char *path, const std::vector<const KBlock *> &B, const std::vector<int> &mv,
                          const std::vector<int> &nkbas_in, int ipar_out, int kmin_out, const std::vector<double> &lv,
                          const Pass &ps) {
        const int nk = (int)B.size(), nval = (int)lv.size();
        std::vector<int> lmin(nk), lbasis(nk), nkbas(nk);
        int nend = 0;
        for (int i = 0; i < nk; ++i) {  // select :374-380
            lmin[i] = B[i]->k;
            lbasis[i] = B[i]->maxleg + B[i]->lincr - B[i]->k + 1;
            nkbas[i] = (B[i]->ibass / B[i]->iang) * lbasis[i];
            if (!nkbas_in.empty() && nkbas_in[i] != nkbas[i])
                bad(DVR3D_ERR_UNSUPPORTED, "ROTLEV3B: the f-type k = 1 block differs in size from the e-type one");
            nend += nkbas[i];
        }
        FILE *fp = std::fopen(path, "wb");
        if (!fp) bad(DVR3D_ERR_ARG, std::string("cannot open ") + path);
        struct Closer {
            FILE *f;
            ~Closer() { std::fclose(f); }
        } closer{fp};
        RecordWriter w{fp};
        for (int v : {idia, ipar_out, ndvr, nmax, h[4], jrot, kmin_out, nval}) w.i4(v);
        w.end();
        w.put(flags.first, 56);  // zembed, zmors1, zmors2, xmass, g1, g2, zncor (zquad2 dropped)
        w.end();
        for (double v : morse) w.r8(v);
        w.end();
        w.i4(nend);
        for (int v : lmin) w.i4(v);
        for (int v : lbasis) w.i4(v);
        for (int v : nkbas) w.i4(v);
        w.end();
        for (double v : rgrid) w.r8(v);
        w.end();
        w.i4(nval);
        w.end();
        for (double v : lv) w.r8(v);
        w.end();
        std::vector<double> dh;
        for (int i = 0; i < nk; ++i) {
            const KBlock &b = *B[i];
            const int mvi = mv[i], nang = lbasis[i], nrad = b.ibass / b.iang;
            if (mvi <= 0) continue;
            if (nang > b.maxleg + 1) bad(DVR3D_ERR_ARG, "wavefunction file: angular basis larger than its transform");
            // tofbr / jtran: B (nang x nrad mv) = P'' (nang x iang) V (iang x nrad mv), P''(j, kk) =
            // pleg(j, kk-th kept angle)
            std::vector<double> pk((size_t)nang * b.iang, 0.0);
            int kk = 0;
            for (int a = 0; a < b.nang; ++a) {
                if (b.iv[a] == 0) continue;
                if (kk >= b.iang) bad(DVR3D_ERR_ARG, "wavefunction file: more kept angles than iang");
                for (int j = 0; j < nang; ++j) pk[(size_t)kk * nang + j] = b.pleg[(size_t)a * (b.maxleg + 1) + j];
                ++kk;
            }
            if (kk != b.iang) bad(DVR3D_ERR_ARG, "wavefunction file: kept angles differ from iang");
            double *Pd = ctx->arena.get_t<double>("rt_tp", pk.size());
            CK(cudaMemcpyAsync(Pd, pk.data(), sizeof(double) * pk.size(), cudaMemcpyHostToDevice, st));
            double *V = upload_vectors(b, mvi, "rt_c1");
            double *Bm = ctx->arena.get_t<double>("rt_tb", (size_t)nkbas[i] * mvi);
            double *D = ctx->arena.get_t<double>("rt_td", (size_t)nkbas[i] * nval);
            launch_dgemm(false, false, nang, nrad * mvi, b.iang, 1.0, Pd, nang, V, b.iang, 0.0, Bm, nang, st);
            CK(cudaGetLastError());
            // D (nkbas x nval) = B (nkbas x mv) C, C = rows off[i] .. of the eigenvectors
            launch_dgemm(false, false, nkbas[i], nval, mvi, 1.0, Bm, nkbas[i], ps.Z + ps.off[i], ps.ldz, 0.0, D, nkbas[i],
                         st);
            CK(cudaGetLastError());
            dh.resize((size_t)nkbas[i] * nval);
            CK(cudaMemcpyAsync(dh.data(), D, sizeof(double) * dh.size(), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            w.put(dh.data(), sizeof(double) * dh.size());
            w.end();
        }
    };
    // ---- first (or only) pass: e parity for KMIN >= 1, f parity for KMIN = 0
    std::vector<const KBlock *> chain;
    for (auto &b : kb) chain.push_back(&b);
    const bool ztran = kvec_path && kvec_path[0];
    const Pass pe = solve_chain(chain, mvib, ipar0, neval, ztran, levels, "e");
    info.nbass = nbass;
    info.nblk = nblk;
    info.neval = neval;
    info.mvib = mvib;
    if (ztran) write_kvec(kvec_path, chain, mvib, {}, ipar0, kmin == 2 ? 1 : kmin, levels, pe);
    // ---- printed tables (dgrot :1767-1769, :1795-1799)
    table.clear();
    char ln[160];
    auto print_pass = [&](const std::vector<double> &lv, int nb, bool epar) {
        std::snprintf(ln, sizeof(ln), "\n     J =%3d rotational state,%7d basis functions\n", jrot, nb);
        table += ln;
        table += epar ? "            e parity, symmetric |jk> + |j-k> functions in basis\n"
                      : "            f parity, anti-symmetric |jk> - |j-k> functions in basis\n";
        std::snprintf(ln, sizeof(ln), "\n\n     lowest%4d eigenvalues in Hartrees\n\n", (int)lv.size());
        table += ln;
        auto rows = [&](const std::vector<double> &v) {
            for (size_t i = 0; i < v.size(); ++i) {
                table += fmt_d(v[i], 24, 12);
                if (i % 5 == 4 || i + 1 == v.size()) table += "\n\n";
            }
        };
        rows(lv);
        std::vector<double> cm(lv.size());
        for (size_t i = 0; i < lv.size(); ++i) cm[i] = lv[i] * 2.19474624e5 - rd.ezero;
        std::snprintf(ln, sizeof(ln), "\n\n     lowest%4d eigenvalues in wavenumbers relative to ezero =", (int)lv.size());
        table += ln;
        table += fmt_d(rd.ezero, 24, 12) + "\n\n";
        rows(cm);
    };
    print_pass(levels, nbass, kmin >= 1);
    if (kmin != 2) return;
    // ---- KMIN = 2, second pass (vrmain :600-660): f parity, k = 1..J, with the f-type k = 1
    // block in place of the e-type one; its Coriolis blocks with k = 2, 3 are formed anew
    // (solrt :1529-1617, ip = 1 - ipar), those among k >= 2 are the same as in the first pass
    const int nbf = nbass - mvib[0];
    const int nevf = std::min(neval2, nbf);
    const bool ztran2 = kvec2_path && kvec2_path[0];
    if (jrot == 1) {
        // J = 1 f: the k = 1 f block alone, its levels and vectors as they are (dstore1 :2051-2173)
        const int nv = std::min(nevf, kf1.meval);
        levels_f->assign(kf1.ev.begin(), kf1.ev.begin() + nv);
        if (ztran2) {
            FILE *fp = std::fopen(kvec2_path, "wb");
            if (!fp) bad(DVR3D_ERR_ARG, std::string("cannot open ") + kvec2_path);
            struct Closer {
                FILE *f;
                ~Closer() { std::fclose(f); }
            } closer{fp};
            RecordWriter w{fp};
            const int ipf = 1 - ipar0, idvr = kb[nblk - 1].nang;
            for (int v : {idia, ipf, idvr, nmax, h[4], jrot, 0, nv}) w.i4(v);
            w.end();
            w.put(flags.first, 56);
            w.end();
            for (double v : morse) w.r8(v);
            w.end();
            const int max2d = nmax * (nmax + 1 - 2 * ipf) / 2, mbass = idvr * max2d;
            for (int v : {mbass, 0, idvr, mbass}) w.i4(v);
            w.end();
            for (double v : rgrid) w.r8(v);
            w.end();
            const double *xa = f.vec(kf1.xalf_rec, 0);
            const size_t nxa = std::min<size_t>((size_t)idvr, f.rec[kf1.xalf_rec].second / 8);
            w.put(xa, 8 * nxa);
            w.end();
            for (int v : {kf1.k, kf1.maxleg, kf1.nang}) w.i4(v);
            w.end();
            w.put(kf1.pleg.data(), 8 * (size_t)kf1.nang * ndvr > 8 * kf1.pleg.size() ? 8 * kf1.pleg.size()
                                                                                       : 8 * (size_t)kf1.nang * ndvr);
            w.end();
            w.i4(kf1.iang);
            w.i4(kf1.ibass);
            w.end();
            for (int v : kf1.iv) w.i4(v);
            w.end();
            w.i4(nv);
            w.end();
            w.put(kf1.ev.data(), 8 * (size_t)nv);
            w.end();
            for (int l = 0; l < nv; ++l) {
                w.put(f.vec(kf1.vec0 + l, (size_t)kf1.ibass), 8 * (size_t)kf1.ibass);
                w.end();
            }
        }
    } else {
        std::vector<const KBlock *> fchain{&kf1};
        std::vector<int> mvf{std::min(mvib[1], std::min(kf1.ibass, kf1.meval))};
        if (mvf[0] != mvib[1]) bad(DVR3D_ERR_ARG, "wavefunction file: the f-type k = 1 block holds too few vectors");
        std::vector<int> nkb_ref{(kb[1].ibass / kb[1].iang) * (kb[1].maxleg + kb[1].lincr - kb[1].k + 1)};
        for (int i = 2; i < nblk; ++i) {
            fchain.push_back(&kb[i]);
            mvf.push_back(mvib[i]);
            nkb_ref.push_back((kb[i].ibass / kb[i].iang) * (kb[i].maxleg + kb[i].lincr - kb[i].k + 1));
        }
        const Pass pf = solve_chain(fchain, mvf, 1 - ipar0, nevf, ztran2, *levels_f, "f");
        if (pf.nb != nbf) bad(DVR3D_ERR_ARG, "ROTLEV3B: f basis size mismatch");
        if (ztran2) write_kvec(kvec2_path, fchain, mvf, nkb_ref, 1 - ipar0, 0, *levels_f, pf);
    }
    print_pass(*levels_f, nbf, false);
}

}  // namespace dvr3d
