// rotlev3_oracle.cpp -- CPU restatement of the reference's program ROTLEV3
// (source/rotlev3.f90): the second variational step for embeddings with z along r1 or r2
// (Jacobi coordinates, IDIA = 1, 2, and Radau with the z axis on a bond). The k blocks of a
// first-step (ZTRAN) wavefunction file are coupled only to their neighbours; each block's
// vectors are taken from the angular DVR to associated Legendre functions (jtran :839-905) and
// the Coriolis elements summed over the FBR functions two neighbouring blocks share, at every
// radial point (solrt :671-837). In-core Hamiltonian (loadh :907-973, ZDCORE), lowest NEVAL
// levels (dgrot :1046-1199), the vectors transformed back for DIPOLE3 (dstore :1201-1342) and
// the J = 1 f special case (dstore1 :1344-1476); KMIN = 2 does the e set and then the f set, the
// Hamiltonian without its k = 0 block (vrmain :600-660).
//
// TEST INFRASTRUCTURE ONLY: the parity checker of the product's dvr3d_b200_rotlev3. It follows
// the reference loop by loop (the rank-1 updates of solrt, the sums of jtran in their order).
// Nothing in the product links or calls it.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../include/dvr3d_b200.h"
#include "dvr3d_oracle.h"

namespace {

struct R3Fail {
    int code;
};
[[noreturn]] void r3fail(int code) { throw R3Fail{code}; }

// A sequential unformatted file with its records addressable by position (the reference reads
// it front to back and rewinds; the same records are taken here by index).
struct R3File {
    std::vector<unsigned char> b;
    std::vector<std::pair<size_t, size_t>> rec;
    explicit R3File(const char *path) {
        FILE *fp = std::fopen(path, "rb");
        if (!fp) r3fail(DVR3D_ERR_ARG);
        std::fseek(fp, 0, SEEK_END);
        const long n = std::ftell(fp);
        std::fseek(fp, 0, SEEK_SET);
        b.resize((size_t)std::max(n, 0L));
        const size_t got = n > 0 ? std::fread(b.data(), 1, (size_t)n, fp) : 0;
        std::fclose(fp);
        if (got != b.size()) r3fail(DVR3D_ERR_ARG);
        size_t p = 0;
        while (p + 8 <= b.size()) {
            int32_t m;
            std::memcpy(&m, &b[p], 4);
            if (m < 0 || p + 8 + (size_t)m > b.size()) r3fail(DVR3D_ERR_ARG);
            rec.emplace_back(p + 4, (size_t)m);
            p += 8 + (size_t)m;
        }
    }
    // record i, at least `need` bytes long (a shorter record is the reference's read error)
    const unsigned char *at(size_t i, size_t need) const {
        if (i >= rec.size() || rec[i].second < need) r3fail(DVR3D_ERR_ARG);
        return &b[rec[i].first];
    }
    size_t len(size_t i) const {
        if (i >= rec.size()) r3fail(DVR3D_ERR_ARG);
        return rec[i].second;
    }
    std::vector<int> ints(size_t i, size_t n) const {
        std::vector<int> v(n);
        if (n) std::memcpy(v.data(), at(i, 4 * n), 4 * n);
        return v;
    }
    std::vector<double> dbls(size_t i, size_t n) const {
        std::vector<double> v(n);
        if (n) std::memcpy(v.data(), at(i, 8 * n), 8 * n);
        return v;
    }
};

void r3put(FILE *fp, const void *p, size_t n) {
    const int32_t m = (int32_t)n;
    std::fwrite(&m, 4, 1, fp);
    if (n) std::fwrite(p, 1, n, fp);
    std::fwrite(&m, 4, 1, fp);
}

// One k block of the first-step file as select and solrt read it.
struct R3Block {
    int k = 0, maxleg = 0, idvr = 0, lincr = 0, meval = 0;
    size_t rec0 = 0;            // record index of the block's xalf; kz line +1, pleg +2, meval +3,
                                // energies +4, vectors +5 ..
    std::vector<double> pleg;   // (maxleg + 1) x idvr
    std::vector<double> evib;   // meval levels (hartree)
    int jst = 0, nang = 0, maxlg = 0;
    std::vector<double> coef;   // jtran: (nang nrad) x mvib, column-major
};

// The deck: namelist PRT (its flags do not change the numbers here), then
// NVIB NEVAL KMIN IBASS NEVAL2 (12i5), the title (9a8) and the optional EZERO (f20.0).
struct R3Cards {
    int nvib = 0, neval = 0, kmin = 0, ibass = 0, neval2 = 0;
};

R3Cards r3_cards(const char *text) {
    std::vector<std::string> ln(1);
    for (const char *c = text; *c; ++c) {
        if (*c == '\n') ln.emplace_back();
        else if (*c != '\r') ln.back() += *c;
    }
    size_t i = 0;
    while (i < ln.size() && ln[i].find('/') == std::string::npos) ++i;
    ++i;
    if (i >= ln.size()) r3fail(DVR3D_ERR_DECK);
    auto i5 = [&](int f) {
        const std::string &s = ln[i];
        if ((size_t)(5 * f) >= s.size()) return 0;
        const std::string t = s.substr(5 * f, 5);
        const size_t a = t.find_first_not_of(' ');
        return a == std::string::npos ? 0 : std::atoi(t.c_str() + a);
    };
    R3Cards c;
    c.nvib = i5(0);
    c.neval = i5(1);
    c.kmin = i5(2);
    c.ibass = i5(3);
    c.neval2 = i5(4);
    return c;
}

}  // namespace

namespace {

struct R3Out {
    std::vector<double> e, f;  // levels (hartree): the first (or only) set, the KMIN = 2 f set
};

int rotlev3_run(const char *deck_text, const char *wave_path, const char *kvec_path, const char *kvec2_path,
                R3Out &out) {
    const R3Cards cd = r3_cards(deck_text);
    int nvib = cd.nvib, neval = cd.neval, ibass = cd.ibass, neval2 = cd.neval2;
    const int kmin = cd.kmin;
    // ---- insize :124-200: the file's header records
    const R3File F(wave_path);
    const std::vector<int> h = F.ints(0, 9);
    const int idia = h[0], ipar = h[1], npntt = h[2], npnt1 = h[3], npnt2 = h[4], jrot = h[5], kmin0 = h[6];
    const int meval0 = h[7];
    const unsigned char *fl = F.at(1, 60);
    auto flag = [&](int o) {
        int32_t v;
        std::memcpy(&v, fl + o, 4);
        return v != 0;
    };
    const bool zembed = flag(0), z1da = flag(52);
    bool zquad2 = flag(56);
    if (idia == -2 || jrot <= 0) r3fail(DVR3D_ERR_UNSUPPORTED);  // symmetrised Radau: ROTLEV3B
    if (z1da) r3fail(DVR3D_ERR_UNSUPPORTED);                     // DVR1DA input vectors
    if (kmin < 0 || kmin > 2) r3fail(DVR3D_ERR_ARG);
    if (kmin > 0 && kmin0 != 1) r3fail(DVR3D_ERR_ARG);           // :287-288 (stop 960)
    const int mbass = npnt1 * npnt2 * npntt;
    nvib = std::min(nvib, meval0);
    const int nblk = jrot + (kmin > 0 ? 1 : 0);
    int nbass = nblk * nvib;
    if (ibass > 0) nbass = std::min(nbass, ibass);
    if (neval <= 0) neval = 10;
    neval = std::min(neval, nbass);
    if (neval2 <= 0) neval2 = neval;
    if (!zembed) zquad2 = true;
    if (!zquad2) r3fail(DVR3D_ERR_UNSUPPORTED);  // r^-2 on the full r2 grid (zquad2 = F)
    const int jdia = std::max(idia, 1), nrad = npnt1 * npnt2;
    // records: 2 Morse constants, 3 r^-2 term (solrt :718), 4 r1, 5 r2, then the k blocks
    const std::vector<double> morse = F.dbls(2, 6);
    const int nlim = zembed ? npnt2 : npnt1;
    const std::vector<double> rm2 = F.dbls(3, (size_t)nlim);
    const std::vector<double> r1 = F.dbls(4, npnt1), r2 = F.dbls(5, npnt2);
    // ---- select :301-480: the blocks in file order, the k = 0 block skipped for KMIN = 0
    std::vector<R3Block> blk;
    std::vector<size_t> fblock;  // record index of every block of the file, in order
    {
        size_t ri = 6;
        while (ri < F.rec.size()) {
            fblock.push_back(ri);
            const int me = F.ints(ri + 3, 1)[0];
            ri += 5 + (size_t)std::max(me, 0);
        }
    }
    for (size_t fb = 0; fb < fblock.size() && (int)blk.size() < nblk; ++fb) {
        R3Block B;
        B.rec0 = fblock[fb];
        const std::vector<int> kh = F.ints(B.rec0 + 1, 4);
        B.k = kh[0];
        B.maxleg = kh[1];
        B.idvr = kh[2];
        B.lincr = kh[3];
        if (B.k == 0 && kmin == 0) continue;
        B.pleg = F.dbls(B.rec0 + 2, (size_t)(B.maxleg + 1) * B.idvr);
        B.meval = F.ints(B.rec0 + 3, 1)[0];
        B.evib = F.dbls(B.rec0 + 4, (size_t)B.meval);
        blk.push_back(std::move(B));
    }
    if ((int)blk.size() < nblk) r3fail(DVR3D_ERR_ARG);  // end of file (:900-940)
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
        ipt = ibass;
    }
    nbass = ipt;
    neval = std::min(neval, nbass);
    // ---- jtran :839-905, per block: jstart, nang and the FBR coefficients
    //      coef(j + (mn-1) nang, l) = sum_k dvrvec(k, mn) pleg(jj, k),  l = jstart + (j-1) jdia
    for (int m = 0; m < nblk; ++m) {
        R3Block &B = blk[m];
        B.maxlg = B.maxleg + B.lincr;  // solrt :756-757
        if (B.maxlg % jdia != ipar) B.maxlg -= 1;
        int jstart = B.k, jj0 = -jdia;
        if (jstart % jdia != ipar) {
            jj0 += 1;
            jstart += 1;
        }
        B.jst = jstart;
        B.nang = (B.maxleg + B.lincr - jstart) / jdia + 1;
    }
    // the flags record as dstore writes it: zembed .. g2, then .false. (:1271)
    std::vector<unsigned char> flags(56, 0);
    std::memcpy(flags.data(), fl, 52);
    auto header = [&](FILE *fp, int kmin1, int nvl) {
        const int hd[8] = {idia, ipar, npntt, npnt1, npnt2, jrot, kmin1, nvl};
        r3put(fp, hd, sizeof(hd));
        r3put(fp, flags.data(), flags.size());
        r3put(fp, morse.data(), 8 * morse.size());
    };
    // dstore1 :1344-1476 (itra = 2): the J = 1 f set is the file's second k block (k = 1) as the
    // first step left it: its levels and its DVR vectors (the first nkbas amplitudes of each)
    // under a header of a single-block file. The reference takes lmin, lbasis, nkbas from the
    // scratch record jtran wrote for that block; they are formed here from the block itself.
    auto dstore1 = [&](const char *path, int nvl, std::vector<double> &lev) {
        if (fblock.size() < 2) r3fail(DVR3D_ERR_ARG);  // the reference reads past the file's end
        R3Block B;
        B.rec0 = fblock[1];
        const std::vector<int> kh = F.ints(B.rec0 + 1, 4);
        B.k = kh[0];
        B.maxleg = kh[1];
        B.idvr = kh[2];
        B.lincr = kh[3];
        B.meval = F.ints(B.rec0 + 3, 1)[0];
        if (B.meval < nvl) r3fail(DVR3D_ERR_ARG);
        lev = F.dbls(B.rec0 + 4, (size_t)nvl);
        if (!path) return;
        int jstart = B.k;
        if (jstart % jdia != ipar) jstart += 1;
        const int nang = (B.maxleg + B.lincr - jstart) / jdia + 1, nkbas = nang * nrad;
        FILE *fp = std::fopen(path, "wb");
        if (!fp) r3fail(DVR3D_ERR_ARG);
        header(fp, 0, nvl);
        const int r4[4] = {nkbas, jstart, nang, nkbas};
        r3put(fp, r4, sizeof(r4));
        r3put(fp, r1.data(), 8 * r1.size());
        r3put(fp, r2.data(), 8 * r2.size());
        const size_t nx = std::min((size_t)npntt, F.len(B.rec0) / 8);
        r3put(fp, F.at(B.rec0, 8 * nx), 8 * nx);
        r3put(fp, kh.data(), 16);
        const size_t nl = (size_t)(B.maxleg + 1) * B.idvr;
        r3put(fp, F.at(B.rec0 + 2, 8 * nl), 8 * nl);
        r3put(fp, &nvl, 4);
        r3put(fp, lev.data(), 8 * (size_t)nvl);
        for (int i = 0; i < nvl; ++i) r3put(fp, F.at(B.rec0 + 5 + i, 8 * (size_t)nkbas), 8 * (size_t)nkbas);
        std::fclose(fp);
    };
    if (jrot == 1 && kmin == 0) {  // vrmain :504-508: J = 1 f, no Hamiltonian; the set goes to KVEC2
        dstore1(kvec2_path, neval, out.e);
        return DVR3D_OK;
    }
    for (int m = 0; m < nblk; ++m) {
        R3Block &B = blk[m];
        const int mv = mvib[m];
        if (mv <= 0) continue;
        int jj0 = -jdia;
        if (B.k % jdia != ipar) jj0 += 1;
        const size_t ib2 = (size_t)B.idvr * nrad, nk = (size_t)B.nang * nrad;
        if (jj0 + jdia * B.nang > B.maxleg) r3fail(DVR3D_ERR_ARG);  // pleg has rows 0..maxleg
        B.coef.assign(nk * mv, 0.0);
        std::vector<double> sumk(nrad);
        for (int l = 0; l < mv; ++l) {
            const std::vector<double> dv = F.dbls(B.rec0 + 5 + l, ib2);
            int jj = jj0;
            for (int j = 0; j < B.nang; ++j) {
                std::fill(sumk.begin(), sumk.end(), 0.0);
                jj += jdia;
                for (int k = 0; k < B.idvr; ++k) {
                    const double p = B.pleg[(size_t)jj + (size_t)k * (B.maxleg + 1)];
                    for (int mn = 0; mn < nrad; ++mn) sumk[mn] += dv[(size_t)k + (size_t)mn * B.idvr] * p;
                }
                for (int mn = 0; mn < nrad; ++mn) B.coef[(size_t)j + (size_t)mn * B.nang + l * nk] = sumk[mn];
            }
        }
    }
    // ---- solrt :671-837 and loadh :907-973: the first-step energies on the diagonal, and for
    //      every pair of neighbouring blocks (k-1, k) the Coriolis block
    //      offdg(a, b) += cor coef_k(j, a) coef_{k-1}(i, b),  cor = cjlp(l) rm2(r),
    //      cjlp = -sqrt((l(l+1) - k(k-1)) (J(J+1) - k(k-1))) (times sqrt2 for k = 1),
    //      over the l both blocks hold at every radial point (ijump / jjump line them up)
    std::vector<int> off(nblk + 1, 0);
    for (int m = 0; m < nblk; ++m) off[m + 1] = off[m] + mvib[m];
    if (off[nblk] != nbass) r3fail(DVR3D_ERR_ARG);
    std::vector<double> H((size_t)nbass * nbass, 0.0);
    for (int m = 0; m < nblk; ++m)
        for (int i = 0; i < mvib[m]; ++i) H[(size_t)(off[m] + i) * (nbass + 1)] = blk[m].evib[i];
    const int jjp1 = jrot * (jrot + 1);
    const double sqrt2 = 1.4142135623731;  // solrt's DATA constant
    for (int m = 1; m < nblk; ++m) {
        const int mv1 = mvib[m - 1], mv2 = mvib[m];
        if (mv1 * mv2 == 0) continue;
        const R3Block &B1 = blk[m - 1], &B2 = blk[m];
        const int K = (kmin == 0 ? 1 : 0) + m, kkp1 = K * (K - 1);
        const int ijump = (B2.jst - B1.jst) / jdia, jjump = B2.maxlg / jdia - B1.maxlg / jdia;
        const size_t nk1 = (size_t)B1.nang * nrad, nk2 = (size_t)B2.nang * nrad;
        std::vector<double> offdg((size_t)mv2 * mv1, 0.0);
        int ii = 0, j = 0;
        for (int n1 = 0; n1 < npnt2; ++n1)
            for (int m1 = 0; m1 < npnt1; ++m1) {
                ii += ijump;
                for (int l1 = B2.jst; l1 <= B1.maxlg; l1 += jdia) {
                    double cjlp = -std::sqrt((double)((l1 * (l1 + 1) - kkp1) * (jjp1 - kkp1)));
                    if (K == 1) cjlp = sqrt2 * cjlp;
                    ++ii;
                    ++j;
                    if ((size_t)ii > nk1 || (size_t)j > nk2) r3fail(DVR3D_ERR_ARG);
                    const double cor = cjlp * (zembed ? rm2[n1] : rm2[m1]);
                    // dger(mv2, mv1, cor, coef2(j, 1), mbass, coef1(i, 1), mbass, offdg, mv2)
                    for (int b = 0; b < mv1; ++b) {
                        const double t = cor * B1.coef[(size_t)(ii - 1) + b * nk1];
                        for (int a = 0; a < mv2; ++a) offdg[a + (size_t)b * mv2] += B2.coef[(size_t)(j - 1) + a * nk2] * t;
                    }
                }
                j += jjump;
            }
        for (int b = 0; b < mv1; ++b)
            for (int a = 0; a < mv2; ++a) {
                const size_t r = off[m - 1] + b, c = off[m] + a;
                H[r + c * nbass] = H[c + r * nbass] = offdg[a + (size_t)b * mv2];
            }
    }
    // dstore :1201-1342: per block D = B C (B the block's jtran coefficients, C its rows of the
    // eigenvectors), D held with leading dimension MBASS and its first nkbas nval elements
    // written (the reference's outrow of d; the same as the block's columns when nkbas = MBASS,
    // i.e. every block has the full angular basis, ZLADD)
    auto dstore = [&](const char *path, int m0, int kmin1, int nvl, const std::vector<double> &vec, int nb,
                      const std::vector<double> &ev) {
        FILE *fp = std::fopen(path, "wb");
        if (!fp) r3fail(DVR3D_ERR_ARG);
        header(fp, kmin1, nvl);
        std::vector<int> r4{0}, lb, nkb;
        for (int m = m0; m < nblk; ++m) {
            r4.push_back(blk[m].jst);
            lb.push_back(blk[m].nang);
            nkb.push_back(blk[m].nang * nrad);
            r4[0] += blk[m].nang * nrad;
        }
        r4.insert(r4.end(), lb.begin(), lb.end());
        r4.insert(r4.end(), nkb.begin(), nkb.end());
        r3put(fp, r4.data(), 4 * r4.size());
        r3put(fp, r1.data(), 8 * r1.size());
        r3put(fp, r2.data(), 8 * r2.size());
        r3put(fp, &nvl, 4);
        r3put(fp, ev.data(), 8 * (size_t)nvl);
        int mbeg = 0;
        for (int m = m0; m < nblk; ++m) {
            const int mv = mvib[m];
            const size_t nk = (size_t)blk[m].nang * nrad;
            std::vector<double> d(nk * nvl, 0.0);
            if (mv > 0)
                for (size_t e = 0; e < d.size(); ++e) {
                    const size_t r = e % (size_t)mbass, c = e / (size_t)mbass;
                    if (r >= nk) continue;
                    double s = 0.0;
                    for (int l = 0; l < mv; ++l) s += vec[(size_t)(mbeg + l) + c * nb] * blk[m].coef[r + l * nk];
                    d[e] = s;
                }
            mbeg += mv;
            r3put(fp, d.data(), 8 * d.size());
        }
        std::fclose(fp);
    };
    // ---- dgrot :1046-1199: the lowest NEVAL levels of the in-core Hamiltonian
    std::vector<double> V = H, ev(nbass);
    if (oracle_dsyev_lower(V.data(), nbass, ev.data()) != DVR3D_OK) r3fail(DVR3D_ERR_NOCONV);
    out.e.assign(ev.begin(), ev.begin() + neval);
    if (kvec_path) dstore(kvec_path, 0, kmin == 2 ? 1 : kmin, neval, V, nbass, out.e);
    if (kmin <= 1) return DVR3D_OK;
    // ---- the f set (vrmain :600-660): the Hamiltonian without its first (k = 0) block
    const int nbf = nbass - mvib[0], nevf = std::min(neval2, nbf);
    if (jrot == 1) {
        dstore1(kvec2_path, nevf, out.f);
        return DVR3D_OK;
    }
    std::vector<double> Vf((size_t)nbf * nbf), evf(nbf);
    for (int c = 0; c < nbf; ++c)
        for (int r = 0; r < nbf; ++r) Vf[r + (size_t)c * nbf] = H[(mvib[0] + r) + (size_t)(mvib[0] + c) * nbass];
    if (oracle_dsyev_lower(Vf.data(), nbf, evf.data()) != DVR3D_OK) r3fail(DVR3D_ERR_NOCONV);
    out.f.assign(evf.begin(), evf.begin() + nevf);
    if (kvec2_path) dstore(kvec2_path, 1, 0, nevf, Vf, nbf, out.f);
    return DVR3D_OK;
}

}  // namespace

extern "C" int oracle_rotlev3(const char *deck_text, const char *wave_path, const char *kvec_path,
                              const char *kvec2_path, double *levels, int cap, int *nlev, double *levels_f, int cap_f,
                              int *nlev_f) {
    if (!deck_text || !wave_path || !nlev) return DVR3D_ERR_ARG;
    try {
        R3Out o;
        const int rc = rotlev3_run(deck_text, wave_path, kvec_path && kvec_path[0] ? kvec_path : nullptr,
                                   kvec2_path && kvec2_path[0] ? kvec2_path : nullptr, o);
        if (rc != DVR3D_OK) return rc;
        *nlev = (int)o.e.size();
        if (levels) {
            if (cap < (int)o.e.size()) return DVR3D_ERR_BUFFER;
            std::copy(o.e.begin(), o.e.end(), levels);
        }
        if (nlev_f) *nlev_f = (int)o.f.size();
        if (levels_f && !o.f.empty()) {
            if (cap_f < (int)o.f.size()) return DVR3D_ERR_BUFFER;
            std::copy(o.f.begin(), o.f.end(), levels_f);
        }
        return DVR3D_OK;
    } catch (const R3Fail &f) {
        return f.code;
    }
}
