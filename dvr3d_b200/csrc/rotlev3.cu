// rotlev3.cu -- the second variational step for J > 0 with the z axis along r1 or r2 (Jacobi
// coordinates, IDIA = 1 or 2, and unsymmetrised Radau): the reference's ROTLEV3
// (source/rotlev3.f90).
//
// Input: the first step's wavefunction file (ZROT, ZTRAN) and ROTLEV3's deck. With z along a
// bond only k and k +- 1 couple. The reference takes every block's vectors from the angular DVR
// to associated Legendre functions (jtran :839-905) and, at every radial point, adds one rank-1
// update per Legendre function l that blocks k-1 and k share (solrt :671-837):
//     offdg(a, b) += cjlp(l) rm2(r) coef_k(l, r; a) coef_{k-1}(l, r; b),
//     cjlp(l) = -sqrt((l(l+1) - k(k-1)) (J(J+1) - k(k-1))), times sqrt2 for k = 1.
// Here both are DMMA GEMMs (gemm64):
//   * jtran per block: coef (nang x nrad mvib) = P (nang x idvr) V (idvr x nrad mvib), P the
//     block's normalised Legendre functions times DVR weights at its points, V its first-step
//     vectors as the file holds them;
//   * the Coriolis block: one gather kernel lays out, for every (radial point, shared l), the
//     row of coef_{k-1} scaled by cjlp rm2 and the row of coef_k; offdg = G_k^T G_{k-1}, one
//     GEMM with K = nrad x (number of shared l).
// The Hamiltonian (loadh's in-core form :907-973) is assembled on the device and its lowest
// NEVAL levels come from the dense FP64 eigensolver (dgrot :1046-1199 takes them with DSYEVX, or
// with the iterative F02FJF when ZDCORE is off: the same levels). KMIN = 2 does the e set and
// then the f set: the same Hamiltonian without its k = 0 block (vrmain :600-660). ZTRAN writes
// the vectors back in the first step's FBR basis (dstore :1201-1342: D = coef C per block, one
// GEMM each); J = 1 f copies the file's k = 1 block (dstore1 :1344-1476).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
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

[[noreturn]] void bad3(int code, const std::string &m) { throw HostError{code, m}; }

unsigned grid256(long long n) { return (unsigned)std::max<long long>(1, std::min<long long>((n + 255) / 256, 8192)); }

__global__ void r3_diag_kernel(const double *dg, int n, double *H, long long ldh) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        H[i * ldh + i] = dg[i];
}

// The Coriolis operands of one block pair. Row t = r nc + c of both (r the radial point, r1
// fastest; c the c-th shared Legendre function): G1[t, b] = cjlp[c] rm2[r1 or r2 of r]
// coef1[r nang1 + ijump + c, b] and G2[t, a] = coef2[r nang2 + c, a] (solrt's ii and j).
__global__ void r3_gather_kernel(const double *coef1, long long nk1, int nang1, int ijump, int mv1,
                                 const double *coef2, long long nk2, int nang2, int mv2, const double *cjlp,
                                 const double *rm2, int npnt1, int zembed, int nrad, int nc, double *G1,
                                 double *G2) {
    const long long K = (long long)nrad * nc, mx = (long long)(mv1 > mv2 ? mv1 : mv2);
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < K * mx;
         e += (long long)gridDim.x * blockDim.x) {
        const long long t = e % K, col = e / K;
        const int r = (int)(t / nc), c = (int)(t % nc);
        if (col < mv1) {
            const double cor = cjlp[c] * rm2[zembed ? r / npnt1 : r % npnt1];
            G1[col * K + t] = cor * coef1[col * nk1 + (long long)r * nang1 + ijump + c];
        }
        if (col < mv2) G2[col * K + t] = coef2[col * nk2 + (long long)r * nang2 + c];
    }
}

// H rows r0.. (block k-1) x columns c0.. (block k) and its transpose from off (n2 x n1).
__global__ void r3_place_kernel(const double *off, int n2, int n1, double *H, long long ldh, int r0, int c0) {
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < (long long)n1 * n2;
         e += (long long)gridDim.x * blockDim.x) {
        const int a = (int)(e % n2), b = (int)(e / n2);
        const double v = off[e];
        H[(long long)(c0 + a) * ldh + (r0 + b)] = v;
        H[(long long)(r0 + b) * ldh + (c0 + a)] = v;
    }
}

// Fortran Dw.d (0.ddddD+ee) and Fw.d
std::string fmt_fd(double v, int w, int d) {
    char buf[64];
    if (v == 0.0) {
        std::snprintf(buf, sizeof(buf), "0.%0*dD+00", d, 0);
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
        std::snprintf(buf, sizeof(buf), "%s0.%0*.0fD%c%02d", v < 0 ? "-" : "", d, rm, ex < 0 ? '-' : '+', std::abs(ex));
    }
    std::string s(buf);
    if ((int)s.size() < w) s = std::string(w - s.size(), ' ') + s;
    return s;
}

// One k block of the file as select / solrt read it.
struct J3Block {
    int k = 0, maxleg = 0, idvr = 0, lincr = 0, meval = 0;
    size_t rec0 = 0;  // xalf; kz line +1, pleg +2, meval +3, energies +4, vectors +5 ..
    std::vector<double> pleg, ev;
    int jst = 0, nang = 0, maxlg = 0, jj0 = 0;
    double *coef = nullptr;  // device: (nang nrad) x mvib
};

}  // namespace

void rotlev3_solve(dvr3d_ctx *ctx, const char *deck_text, const char *wave_path, std::vector<double> &levels,
                   std::vector<double> &levels_f, std::string &text, RotInfo &info, const char *kvec_path,
                   const char *kvec2_path) {
    // ---- the deck: namelist PRT, NVIB NEVAL KMIN IBASS NEVAL2 (12i5), title, EZERO (f20.0)
    std::vector<std::string> ln(1);
    for (const char *c = deck_text; *c; ++c) {
        if (*c == '\n') ln.emplace_back();
        else if (*c != '\r') ln.back() += *c;
    }
    size_t li = 0;
    while (li < ln.size() && ln[li].find('/') == std::string::npos) ++li;
    if (++li >= ln.size()) bad3(DVR3D_ERR_DECK, "ROTLEV3 deck: no NVIB/NEVAL/KMIN card after the namelist");
    auto i5 = [&](int fld) {
        const std::string &s = ln[li];
        if ((size_t)(5 * fld) >= s.size()) return 0;
        const std::string t = s.substr(5 * fld, 5);
        const size_t a = t.find_first_not_of(' ');
        return a == std::string::npos ? 0 : std::atoi(t.c_str() + a);
    };
    int nvib = i5(0), neval = i5(1), ibass = i5(3), neval2 = i5(4);
    const int kmin = i5(2);
    double ezero = 0.0;  // vrmain :519-522, the card after the title
    if (li + 2 < ln.size()) {
        std::string t = ln[li + 2].substr(0, std::min<size_t>(20, ln[li + 2].size()));
        for (auto &ch : t)
            if (ch == 'd' || ch == 'D') ch = 'e';
        if (t.find_first_not_of(' ') != std::string::npos) ezero = std::strtod(t.c_str(), nullptr);
    }
    // ---- the file's header (insize :124-128)
    Records f(wave_path);
    auto ints_at = [&](size_t i, size_t n) {
        const auto r = f.at(i);
        if (r.second < 4 * n) bad3(DVR3D_ERR_ARG, "wavefunction file: integer record too short");
        std::vector<int> v(n);
        if (n) std::memcpy(v.data(), r.first, 4 * n);
        return v;
    };
    auto dbls_at = [&](size_t i, size_t n) {
        std::vector<double> v(n);
        if (n) std::memcpy(v.data(), f.vec(i, n), 8 * n);
        return v;
    };
    const std::vector<int> h = ints_at(0, 9);
    const int idia = h[0], ipar = h[1], npntt = h[2], npnt1 = h[3], npnt2 = h[4], jrot = h[5], kmin0 = h[6];
    const int meval0 = h[7];
    const auto flr = f.at(1);
    if (flr.second < 60) bad3(DVR3D_ERR_ARG, "wavefunction file: short flags record");
    auto flag = [&](int o) {
        int32_t v;
        std::memcpy(&v, flr.first + o, 4);
        return v != 0;
    };
    const bool zembed = flag(0);
    if (idia == -2) bad3(DVR3D_ERR_UNSUPPORTED, "ROTLEV3: a symmetrised Radau file (IDIA = -2) is ROTLEV3B's");
    if (jrot <= 0) bad3(DVR3D_ERR_ARG, "ROTLEV3 needs a J > 0 wavefunction file");
    if (flag(52)) bad3(DVR3D_ERR_UNSUPPORTED, "ROTLEV3: DVR1DA-type (FBR) input vectors are not on this path");
    if (zembed && !flag(56)) bad3(DVR3D_ERR_UNSUPPORTED, "ROTLEV3: zquad2 = F (r^-2 on the full r2 grid) is not on this path");
    if (kmin < 0 || kmin > 2) bad3(DVR3D_ERR_ARG, "ROTLEV3: KMIN must be 0, 1 or 2");
    if (kmin > 0 && kmin0 != 1) bad3(DVR3D_ERR_ARG, "ROTLEV3: KMIN > 0 needs a first-step file of KMIN = 1 (insize stop 960)");
    const int mbass = npnt1 * npnt2 * npntt;
    nvib = std::min(nvib, meval0);
    const int nblk = jrot + (kmin > 0 ? 1 : 0);
    int nbass = nblk * nvib;
    if (ibass > 0) nbass = std::min(nbass, ibass);
    if (neval <= 0) neval = 10;
    neval = std::min(neval, nbass);
    if (neval2 <= 0) neval2 = neval;
    const int jdia = std::max(idia, 1), nrad = npnt1 * npnt2;
    const std::vector<double> morse = dbls_at(2, 6);
    const std::vector<double> rm2 = dbls_at(3, (size_t)(zembed ? npnt2 : npnt1));
    const std::vector<double> r1 = dbls_at(4, npnt1), r2 = dbls_at(5, npnt2);
    // ---- select :301-480
    std::vector<size_t> fblock;
    for (size_t ri = 6; ri < f.rec.size();) {
        fblock.push_back(ri);
        ri += 5 + (size_t)std::max(ints_at(ri + 3, 1)[0], 0);
    }
    std::vector<J3Block> blk;
    for (size_t fb = 0; fb < fblock.size() && (int)blk.size() < nblk; ++fb) {
        J3Block B;
        B.rec0 = fblock[fb];
        const std::vector<int> kh = ints_at(B.rec0 + 1, 4);
        B.k = kh[0];
        B.maxleg = kh[1];
        B.idvr = kh[2];
        B.lincr = kh[3];
        if (B.k == 0 && kmin == 0) continue;
        B.pleg = dbls_at(B.rec0 + 2, (size_t)(B.maxleg + 1) * B.idvr);
        B.meval = ints_at(B.rec0 + 3, 1)[0];
        B.ev = dbls_at(B.rec0 + 4, (size_t)B.meval);
        if (B.rec0 + 5 + (size_t)B.meval > f.rec.size()) bad3(DVR3D_ERR_ARG, "wavefunction file: ends inside a k block");
        blk.push_back(std::move(B));
    }
    if ((int)blk.size() < nblk) bad3(DVR3D_ERR_ARG, "wavefunction file holds fewer k blocks than ROTLEV3 needs");
    std::vector<int> mvib(nblk);
    int ipt = 0;
    for (int k = 0; k < nblk; ++k) {
        mvib[k] = std::min(nvib, blk[k].meval);
        ipt += mvib[k];
    }
    if (!(ibass <= 0 || ibass >= ipt)) {  // the IBASS lowest functions (:372-404)
        std::vector<int> iv(nblk, 1);
        int p = 1;
        for (int n = 1; n <= ibass; ++n) {
            while (!(iv[p - 1] <= mvib[p - 1])) p = p + 1;
            double evibr = blk[p - 1].ev[iv[p - 1] - 1];
            int jpt = p;
            for (int j = p + 1; j <= nblk; ++j) {
                if (iv[j - 1] > mvib[j - 1]) continue;
                if (blk[j - 1].ev[iv[j - 1] - 1] >= evibr) continue;
                evibr = blk[j - 1].ev[iv[j - 1] - 1];
                jpt = j;
            }
            iv[jpt - 1] = iv[jpt - 1] + 1;
        }
        for (int i = 0; i < nblk; ++i) mvib[i] = iv[i] - 1;
        ipt = ibass;
    }
    nbass = ipt;
    neval = std::min(neval, nbass);
    info.nbass = nbass;
    info.nblk = nblk;
    info.neval = neval;
    info.mvib = mvib;
    info.offdiag_flops = 0.0;
    for (auto &B : blk) {  // jtran's jstart, nang; solrt's maxlg2
        B.maxlg = B.maxleg + B.lincr;
        if (B.maxlg % jdia != ipar) B.maxlg -= 1;
        B.jst = B.k;
        B.jj0 = -jdia;
        if (B.jst % jdia != ipar) {
            B.jj0 += 1;
            B.jst += 1;
        }
        B.nang = (B.maxleg + B.lincr - B.jst) / jdia + 1;
        if (B.nang < 1 || B.jj0 + jdia * B.nang > B.maxleg)
            bad3(DVR3D_ERR_ARG, "wavefunction file: angular basis larger than its Legendre table");
    }
    // the flags record as dstore writes it: zembed .. g2, then .false. (:1271)
    unsigned char flags[56] = {};
    std::memcpy(flags, flr.first, 52);
    auto open_out = [&](const char *path) {
        FILE *fp = std::fopen(path, "wb");
        if (!fp) bad3(DVR3D_ERR_ARG, std::string("cannot open ") + path);
        return fp;
    };
    auto header = [&](RecordWriter &w, int kmin1, int nvl) {
        for (int v : {idia, ipar, npntt, npnt1, npnt2, jrot, kmin1, nvl}) w.i4(v);
        w.end();
        w.put(flags, 56);
        w.end();
        for (double v : morse) w.r8(v);
        w.end();
    };
    char line[256];
    auto print_levels = [&](const std::vector<double> &lv, bool epar, int nb) {
        std::snprintf(line, sizeof(line), "     J =%3d ROTATIONAL STATE,%7d BASIS FUNCTIONS\n", jrot, nb);
        text += line;
        text += epar ? "            E PARITY, SYMMETRIC |JK> + |J-K> FUNCTIONS IN BASIS\n"
                     : "            F PARITY, ANTI-SYMMETRIC |JK> - |J-K> FUNCTIONS IN BASIS\n";
        if (idia == 2) text += ipar == 0 ? "            EVEN PARITY FUNCTIONS IN BASIS SET\n" : "            ODD PARITY FUNCTIONS IN BASIS SET\n";
        std::snprintf(line, sizeof(line), "\n\n     LOWEST%4d EIGENVALUES IN HARTREES\n\n", (int)lv.size());
        text += line;
        for (size_t i = 0; i < lv.size(); ++i) {
            text += fmt_fd(lv[i], 24, 12);
            if (i % 5 == 4 || i + 1 == lv.size()) text += "\n";
        }
        std::snprintf(line, sizeof(line), "\n\n     Lowest%4d eigenvalues in wavenumbers relative to EZERO =%s\n\n",
                      (int)lv.size(), fmt_fd(ezero, 24, 12).c_str());
        text += line;
        for (size_t i = 0; i < lv.size(); ++i) {
            std::snprintf(line, sizeof(line), "%s%13.5f", i % 10 == 0 ? " " : "", lv[i] * 2.19474624e5 - ezero);
            text += line;
            if (i % 10 == 9 || i + 1 == lv.size()) text += "\n\n";
        }
    };
    // dstore1 :1344-1476 (itra = 2): the J = 1 f set is the file's second k block (k = 1) as the
    // first step left it, under the header of a one-block file; lmin, lbasis, nkbas (from jtran's
    // scratch record in the reference) are formed from the block itself
    auto dstore1 = [&](const char *path, int nvl, std::vector<double> &lv) {
        if (fblock.size() < 2) bad3(DVR3D_ERR_ARG, "ROTLEV3 J = 1 f: the file has no second k block (dstore1 skips the first)");
        const size_t r0 = fblock[1];
        const std::vector<int> kh = ints_at(r0 + 1, 4);
        const int maxleg = kh[1], nidvr = kh[2], lincr = kh[3];
        if (ints_at(r0 + 3, 1)[0] < nvl) bad3(DVR3D_ERR_ARG, "ROTLEV3 J = 1 f: the k = 1 block holds fewer levels than NEVAL");
        lv = dbls_at(r0 + 4, (size_t)nvl);
        if (!path || !path[0]) return;
        int jstart = kh[0];
        if (jstart % jdia != ipar) jstart += 1;
        const int nang = (maxleg + lincr - jstart) / jdia + 1, nkbas = nang * nrad;
        FILE *fp = open_out(path);
        struct Closer {
            FILE *f;
            ~Closer() { std::fclose(f); }
        } closer{fp};
        RecordWriter w{fp};
        header(w, 0, nvl);
        for (int v : {nkbas, jstart, nang, nkbas}) w.i4(v);
        w.end();
        for (double v : r1) w.r8(v);
        w.end();
        for (double v : r2) w.r8(v);
        w.end();
        const size_t nx = std::min((size_t)npntt, f.at(r0).second / 8);
        w.put(f.at(r0).first, 8 * nx);
        w.end();
        for (int v : kh) w.i4(v);
        w.end();
        w.put(f.vec(r0 + 2, (size_t)(maxleg + 1) * nidvr), 8 * (size_t)(maxleg + 1) * nidvr);
        w.end();
        w.i4(nvl);
        w.end();
        w.put(lv.data(), 8 * (size_t)nvl);
        w.end();
        for (int i = 0; i < nvl; ++i) {
            w.put(f.vec(r0 + 5 + i, (size_t)nkbas), 8 * (size_t)nkbas);
            w.end();
        }
    };
    text.clear();
    if (jrot == 1 && kmin == 0) {  // vrmain :504-508: no Hamiltonian; the set goes to KVEC2
        dstore1(kvec2_path, neval, levels);
        print_levels(levels, false, nbass);
        return;
    }
    cudaStream_t st = ctx->stream;
    // ---- jtran: coef (nang x nrad mv) = P (nang x idvr) V (idvr x nrad mv), one GEMM per block
    for (int m = 0; m < nblk; ++m) {
        J3Block &B = blk[m];
        const int mv = mvib[m];
        if (mv <= 0) continue;
        const size_t ib2 = (size_t)B.idvr * nrad, nk = (size_t)B.nang * nrad;
        std::vector<double> P((size_t)B.nang * B.idvr);
        for (int k = 0; k < B.idvr; ++k)
            for (int j = 0; j < B.nang; ++j)
                P[(size_t)k * B.nang + j] = B.pleg[(size_t)(B.jj0 + jdia * (j + 1)) + (size_t)k * (B.maxleg + 1)];
        double *Pd = ctx->arena.get_t<double>("r3_p", P.size());
        double *V = ctx->arena.get_t<double>("r3_v", ib2 * mv);
        B.coef = ctx->arena.get_t<double>("r3_coef" + std::to_string(m), nk * mv);
        CK(cudaMemcpyAsync(Pd, P.data(), sizeof(double) * P.size(), cudaMemcpyHostToDevice, st));
        for (int l = 0; l < mv; ++l)
            CK(cudaMemcpyAsync(V + ib2 * l, f.vec(B.rec0 + 5 + l, ib2), sizeof(double) * ib2, cudaMemcpyHostToDevice, st));
        launch_dgemm(false, false, B.nang, nrad * mv, B.idvr, 1.0, Pd, B.nang, V, B.idvr, 0.0, B.coef, B.nang, st);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(st));  // P and V are reused by the next block
        info.offdiag_flops += 2.0 * B.nang * B.idvr * (double)nrad * mv;
    }
    // ---- the Hamiltonian (solrt + loadh): levels on the diagonal, Coriolis blocks k-1, k
    std::vector<int> off(nblk + 1, 0);
    for (int m = 0; m < nblk; ++m) off[m + 1] = off[m] + mvib[m];
    const long long ldh = (nbass + 7) / 8 * 8;
    double *H = ctx->arena.get_t<double>("r3_h", (size_t)ldh * nbass);
    CK(cudaMemsetAsync(H, 0, sizeof(double) * ldh * nbass, st));
    {
        std::vector<double> dg(nbass);
        for (int m = 0; m < nblk; ++m)
            for (int i = 0; i < mvib[m]; ++i) dg[off[m] + i] = blk[m].ev[i];
        double *dd = ctx->arena.get_t<double>("r3_dg", nbass);
        CK(cudaMemcpyAsync(dd, dg.data(), sizeof(double) * nbass, cudaMemcpyHostToDevice, st));
        DVR3D_COUNT_LAUNCH(1);
        r3_diag_kernel<<<grid256(nbass), 256, 0, st>>>(dd, nbass, H, ldh);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(st));
    }
    const int jjp1 = jrot * (jrot + 1);
    for (int m = 1; m < nblk; ++m) {
        const int mv1 = mvib[m - 1], mv2 = mvib[m];
        if (mv1 * mv2 == 0) continue;
        const J3Block &B1 = blk[m - 1], &B2 = blk[m];
        const int K = (kmin == 0 ? 1 : 0) + m, kkp1 = K * (K - 1);  // solrt's k counter
        const int ijump = (B2.jst - B1.jst) / jdia, jjump = B2.maxlg / jdia - B1.maxlg / jdia;
        std::vector<double> cj;
        for (int l1 = B2.jst; l1 <= B1.maxlg; l1 += jdia) {
            double c = -std::sqrt((double)((l1 * (l1 + 1) - kkp1) * (jjp1 - kkp1)));
            if (K == 1) c = 1.4142135623731 * c;  // solrt's DATA sqrt2
            cj.push_back(c);
        }
        const int nc = (int)cj.size();
        // solrt's counters stay inside both blocks' vectors: ii = r nang1 + ijump + c < nk1 and
        // j = r nang2 + c < nk2 for every radial point r and shared function c
        if (nc == 0) continue;
        if (ijump < 0 || jjump < 0 || ijump + nc != B1.nang || nc + jjump != B2.nang)
            bad3(DVR3D_ERR_ARG, "wavefunction file: the angular bases of neighbouring k blocks do not line up");
        const long long Kd = (long long)nrad * nc;
        double *cjd = ctx->arena.get_t<double>("r3_cj", nc);
        double *rmd = ctx->arena.get_t<double>("r3_rm2", rm2.size());
        double *G1 = ctx->arena.get_t<double>("r3_g1", (size_t)Kd * mv1);
        double *G2 = ctx->arena.get_t<double>("r3_g2", (size_t)Kd * mv2);
        double *O = ctx->arena.get_t<double>("r3_off", (size_t)mv1 * mv2);
        CK(cudaMemcpyAsync(cjd, cj.data(), sizeof(double) * nc, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(rmd, rm2.data(), sizeof(double) * rm2.size(), cudaMemcpyHostToDevice, st));
        DVR3D_COUNT_LAUNCH(1);
        r3_gather_kernel<<<grid256(Kd * std::max(mv1, mv2)), 256, 0, st>>>(
            B1.coef, (long long)B1.nang * nrad, B1.nang, ijump, mv1, B2.coef, (long long)B2.nang * nrad, B2.nang, mv2,
            cjd, rmd, npnt1, zembed ? 1 : 0, nrad, nc, G1, G2);
        CK(cudaGetLastError());
        // offdg (mv2 x mv1) = G2^T G1
        launch_dgemm(true, false, mv2, mv1, (int)Kd, 1.0, G2, Kd, G1, Kd, 0.0, O, mv2, st);
        CK(cudaGetLastError());
        DVR3D_COUNT_LAUNCH(1);
        r3_place_kernel<<<grid256((long long)mv1 * mv2), 256, 0, st>>>(O, mv2, mv1, H, ldh, off[m - 1], off[m]);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(st));
        info.offdiag_flops += 2.0 * (double)Kd * mv1 * mv2;
    }
    // dstore :1201-1342: per block D = coef C (C the block's rows of the eigenvectors), written
    // as the reference's outrow(d, nkbas nval) of a d with leading dimension MBASS: the block's
    // columns one after another when nkbas = MBASS (every block with the full angular basis,
    // ZLADD), otherwise the first nkbas nval elements of that array
    auto dstore = [&](const char *path, int m0, int kmin1, const std::vector<double> &lv, const double *Z,
                      long long ldz) {
        const int nvl = (int)lv.size();
        FILE *fp = open_out(path);
        struct Closer {
            FILE *f;
            ~Closer() { std::fclose(f); }
        } closer{fp};
        RecordWriter w{fp};
        header(w, kmin1, nvl);
        int nend = 0;
        for (int m = m0; m < nblk; ++m) nend += blk[m].nang * nrad;
        w.i4(nend);
        for (int m = m0; m < nblk; ++m) w.i4(blk[m].jst);
        for (int m = m0; m < nblk; ++m) w.i4(blk[m].nang);
        for (int m = m0; m < nblk; ++m) w.i4(blk[m].nang * nrad);
        w.end();
        for (double v : r1) w.r8(v);
        w.end();
        for (double v : r2) w.r8(v);
        w.end();
        w.i4(nvl);
        w.end();
        w.put(lv.data(), 8 * (size_t)nvl);
        w.end();
        std::vector<double> dh, out;
        int zoff = 0;
        for (int m = m0; m < nblk; ++m) {
            const int mv = mvib[m];
            const size_t nk = (size_t)blk[m].nang * nrad;
            out.assign(nk * nvl, 0.0);
            if (mv > 0 && nvl > 0) {
                double *D = ctx->arena.get_t<double>("r3_d", nk * nvl);
                launch_dgemm(false, false, (int)nk, nvl, mv, 1.0, blk[m].coef, (long long)nk, Z + zoff, ldz, 0.0, D,
                             (long long)nk, st);
                CK(cudaGetLastError());
                dh.resize(nk * nvl);
                CK(cudaMemcpyAsync(dh.data(), D, sizeof(double) * dh.size(), cudaMemcpyDeviceToHost, st));
                CK(cudaStreamSynchronize(st));
                for (size_t e = 0; e < out.size(); ++e) {
                    const size_t r = e % (size_t)mbass, c = e / (size_t)mbass;
                    if (r < nk) out[e] = dh[r + c * nk];
                }
            }
            zoff += mv;
            w.put(out.data(), 8 * out.size());
            w.end();
        }
    };
    // ---- dgrot: the lowest NEVAL levels; KMIN = 2 then the f set without the k = 0 block
    const bool ztran = kvec_path && kvec_path[0], ztran2 = kvec2_path && kvec2_path[0];
    const int nbf = nbass - mvib[0], nevf = std::min(neval2, nbf);
    const long long ldf = (nbf + 7) / 8 * 8;
    double *Hf = nullptr;
    if (kmin == 2 && jrot > 1 && nbf > 0) {  // the f Hamiltonian, before the e solve overwrites H
        Hf = ctx->arena.get_t<double>("r3_hf", (size_t)ldf * nbf);
        CK(cudaMemcpy2DAsync(Hf, sizeof(double) * ldf, H + (size_t)mvib[0] * ldh + mvib[0], sizeof(double) * ldh,
                             sizeof(double) * nbf, nbf, cudaMemcpyDeviceToDevice, st));
    }
    auto lowest = [&](double *A, long long lda, int n, int nev, bool vecs, std::vector<double> &lv, const char *tag) {
        double *wv = ctx->arena.get_t<double>(std::string("r3_ev") + tag, nev);
        double *Z = vecs ? ctx->arena.get_t<double>(std::string("r3_z") + tag, (size_t)lda * nev) : nullptr;
        dense_lowest(ctx, A, lda, n, nev, vecs, wv, Z, vecs ? lda : 1, "r3d_", false, nullptr);
        lv.resize(nev);
        CK(cudaMemcpyAsync(lv.data(), wv, sizeof(double) * nev, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        return Z;
    };
    const double *Ze = lowest(H, ldh, nbass, neval, ztran, levels, "e");
    print_levels(levels, kmin >= 1, nbass);
    if (ztran) dstore(kvec_path, 0, kmin == 2 ? 1 : kmin, levels, Ze, ldh);
    levels_f.clear();
    if (kmin <= 1) return;
    if (jrot == 1) {  // vrmain :611-615: J = 1 f is the file's k = 1 block (dstore1)
        dstore1(ztran2 ? kvec2_path : nullptr, nevf, levels_f);
        print_levels(levels_f, false, nbf);
        return;
    }
    if (nbf <= 0) bad3(DVR3D_ERR_ARG, "ROTLEV3 KMIN = 2: no basis functions above the k = 0 block");
    const double *Zf = lowest(Hf, ldf, nbf, nevf, ztran2, levels_f, "f");
    print_levels(levels_f, false, nbf);
    if (ztran2) dstore(kvec2_path, 1, 0, levels_f, Zf, ldf);
}

}  // namespace dvr3d
