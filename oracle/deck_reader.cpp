// deck_reader.cpp -- the oracle's own reader of a DVR3DRJZ job deck.
//
// TEST INFRASTRUCTURE ONLY (part of the CPU checker, see dvr3d_oracle.h). The parity tests
// read every deck twice: the product parses it with dvr3d_b200_parse_deck, the oracle with
// this reader, so a parsing mistake cannot hide by appearing on both sides of a comparison.
//
// It restates the reference's input statements as a sequence of Fortran records:
//   read(5,prt)                        namelist /PRT/, defaults of block data  (:65, :83-168)
//   read(5,5) ncoord                   format 15i5                              (:232-233)
//   read(5,5) npnt2,jrot,...,max3d2    format 15i5 (11 values)                  (:238-239)
//   read(5,500) title                  format 9a8                               (:372-373)
//   read(5,5) fixcos                   format 3f20.0 (setcon's label 5)         (:1042)
//   read(5,5) xmass ; read(5,5) xmassr                                          (:1048-1052)
//   read(5,5) emax1,emax2                                                        (:1057)
//   read(5,5) re1,diss1,we1 ; read(5,5) re2,diss2,we2                           (:1083,:1093)
//   read(5,5,end=55) ezero             format f20.0, optional (diag3d)          (:2751-2753)
// Formatted input follows the Fortran rules for these edit descriptors: a short record is
// padded with blanks, blanks inside a numeric field are ignored (BLANK='NULL'), an empty
// field reads as zero, and an Fw.0 field without a decimal point is an integer value.
#include <cctype>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "dvr3d_oracle.h"

namespace {

struct Records {
    std::vector<std::string> rec;
    size_t pos = 0;
    bool more() const { return pos < rec.size(); }
    const std::string &next() {
        static const std::string empty;
        return pos < rec.size() ? rec[pos++] : (++pos, empty);
    }
};

Records split_records(const char *text) {
    Records r;
    std::string cur;
    for (const char *p = text; *p; ++p) {
        if (*p == '\n') {
            r.rec.push_back(cur);
            cur.clear();
        } else if (*p != '\r') {
            cur.push_back(*p);
        }
    }
    if (!cur.empty()) r.rec.push_back(cur);
    return r;
}

// Characters [col, col+w) of a record, blank padded.
std::string field(const std::string &rec, size_t col, size_t w) {
    std::string f(w, ' ');
    for (size_t i = 0; i < w && col + i < rec.size(); ++i) f[i] = rec[col + i];
    return f;
}

bool read_iw(const std::string &rec, size_t col, size_t w, int *out) {
    std::string s;
    for (char c : field(rec, col, w))
        if (c != ' ' && c != '\t') s.push_back(c);
    if (s.empty()) {
        *out = 0;
        return true;
    }
    char *end = nullptr;
    long v = std::strtol(s.c_str(), &end, 10);
    if (*end) return false;
    *out = (int)v;
    return true;
}

bool read_fw0(const std::string &rec, size_t col, size_t w, double *out) {
    std::string s;
    for (char c : field(rec, col, w)) {
        if (c == ' ' || c == '\t') continue;
        if (c == 'd' || c == 'D' || c == 'e') c = 'E';
        s.push_back(c);
    }
    if (s.empty()) {
        *out = 0.0;
        return true;
    }
    char *end = nullptr;
    double v = std::strtod(s.c_str(), &end);
    if (*end) return false;
    *out = v;
    return true;
}

// Namelist /PRT/ logical variables (the common /outp/ members a deck may set).
int *prt_logical(dvr3d_deck *d, const std::string &name) {
    static const struct {
        const char *name;
        size_t off;
    } vars[] = {
        {"ZPHAM", offsetof(dvr3d_deck, zpham)},   {"ZPRAD", offsetof(dvr3d_deck, zprad)},
        {"ZP1D", offsetof(dvr3d_deck, zp1d)},     {"ZP2D", offsetof(dvr3d_deck, zp2d)},
        {"ZPMIN", offsetof(dvr3d_deck, zpmin)},   {"ZPVEC", offsetof(dvr3d_deck, zpvec)},
        {"ZLMAT", offsetof(dvr3d_deck, zlmat)},   {"ZCUT", offsetof(dvr3d_deck, zcut)},
        {"ZROT", offsetof(dvr3d_deck, zrot)},     {"ZPERP", offsetof(dvr3d_deck, zperp)},
        {"ZEMBED", offsetof(dvr3d_deck, zembed)}, {"ZLIN", offsetof(dvr3d_deck, zlin)},
        {"ZMORS1", offsetof(dvr3d_deck, zmors1)}, {"ZMORS2", offsetof(dvr3d_deck, zmors2)},
        {"ZLADD", offsetof(dvr3d_deck, zladd)},   {"ZTWOD", offsetof(dvr3d_deck, ztwod)},
        {"ZVEC", offsetof(dvr3d_deck, zvec)},     {"ZALL", offsetof(dvr3d_deck, zall)},
        {"ZTHETA", offsetof(dvr3d_deck, ztheta)}, {"ZR2R1", offsetof(dvr3d_deck, zr2r1)},
        {"ZTRAN", offsetof(dvr3d_deck, ztran)},   {"ZQUAD2", offsetof(dvr3d_deck, zquad2)},
        {"ZDIAG", offsetof(dvr3d_deck, zdiag)},   {"ZPFUN", offsetof(dvr3d_deck, zpfun)},
        {"ZX", offsetof(dvr3d_deck, zx)},         {"ZS0", offsetof(dvr3d_deck, zs0)},
        {"ZS1", offsetof(dvr3d_deck, zs1)},
    };
    for (const auto &v : vars)
        if (name == v.name) return reinterpret_cast<int *>(reinterpret_cast<char *>(d) + v.off);
    return nullptr;
}

// Integer unit numbers of /outp/ that a deck may also set; the oracle keeps no files.
bool prt_unit(const std::string &name) {
    static const char *units[] = {"IDIAG1", "IDIAG2", "IOUT1", "IOUT2", "IWAVE", "ILEV", "IEIGS1",
                                  "IVECS1", "IEIGS2", "IVECS2", "IVINT", "IBAND", "INTVEC"};
    for (const char *u : units)
        if (name == u) return true;
    return false;
}

// Reads the namelist group starting at the first non-blank record; a character-level scan:
// name [=] value pairs separated by blanks or commas, ended by '/' or '&END'.
bool read_prt(Records &r, dvr3d_deck *d) {
    while (r.more() && r.rec[r.pos].find_first_not_of(" \t") == std::string::npos) ++r.pos;
    if (!r.more()) return false;
    std::string text;
    bool ended = false;
    while (r.more() && !ended) {
        std::string s = r.next();
        for (char &c : s) c = (char)std::toupper((unsigned char)c);
        const size_t amp_end = s.find("&END");
        size_t cut = s.find('/');
        if (amp_end != std::string::npos && (cut == std::string::npos || amp_end < cut)) cut = amp_end;
        if (cut != std::string::npos) {
            s.resize(cut);
            ended = true;
        }
        text += ' ';
        text += s;
    }
    if (!ended) return false;
    size_t i = text.find('&');
    if (i == std::string::npos || text.compare(i + 1, 3, "PRT") != 0) return false;
    i += 4;
    auto skip_sep = [&]() {
        while (i < text.size() && (text[i] == ' ' || text[i] == ',' || text[i] == '\t')) ++i;
    };
    while (true) {
        skip_sep();
        if (i >= text.size()) break;
        std::string name;
        while (i < text.size() && (std::isalnum((unsigned char)text[i]) || text[i] == '_')) name.push_back(text[i++]);
        skip_sep();
        if (name.empty() || i >= text.size() || text[i] != '=') return false;
        ++i;
        skip_sep();
        std::string val;
        while (i < text.size() && text[i] != ' ' && text[i] != ',' && text[i] != '\t') val.push_back(text[i++]);
        if (int *slot = prt_logical(d, name)) {
            // Fortran logical input: optional leading '.', then T or F decides
            const size_t k = (!val.empty() && val[0] == '.') ? 1 : 0;
            if (k >= val.size() || (val[k] != 'T' && val[k] != 'F')) return false;
            *slot = (val[k] == 'T');
        } else if (!prt_unit(name)) {
            return false;
        }
    }
    return true;
}

void block_data_defaults(dvr3d_deck *d) {
    std::memset(d, 0, sizeof(*d));
    // block data (:158-167); everything not listed there is .false.
    d->zrot = 1;
    d->zladd = 1;
    d->zembed = 1;
    d->zmors2 = 1;
    d->zquad2 = 1;
    d->zdiag = 1;
    d->zr2r1 = 1;
    d->ztheta = 1;
    d->zmors1 = 1;
    d->ncoord = 3;
}

}  // namespace

extern "C" int oracle_parse_deck(const char *text, dvr3d_deck *out) {
    if (!text || !out) return DVR3D_ERR_ARG;
    dvr3d_deck d;
    block_data_defaults(&d);
    Records r = split_records(text);
    if (!read_prt(r, &d)) return DVR3D_ERR_DECK;
    if (!r.more()) return DVR3D_ERR_DECK;
    if (!read_iw(r.next(), 0, 5, &d.ncoord)) return DVR3D_ERR_DECK;
    if (!r.more()) return DVR3D_ERR_DECK;
    {
        const std::string &c = r.next();
        int *dst[11] = {&d.npnt2, &d.jrot, &d.neval, &d.nalf, &d.max2d, &d.max3d,
                        &d.idia,  &d.kmin, &d.npnt1, &d.ipar, &d.max3d2};
        for (int k = 0; k < 11; ++k)
            if (!read_iw(c, 5 * (size_t)k, 5, dst[k])) return DVR3D_ERR_DECK;
    }
    {
        const std::string t = field(r.next(), 0, 72);  // 9a8
        std::memcpy(d.title, t.data(), 72);
        size_t e = 72;
        while (e > 0 && d.title[e - 1] == ' ') --e;
        d.title[e] = '\0';
    }
    auto f3 = [&](double *a, double *b, double *c) {
        const std::string &rec = r.next();
        double tmp;
        return read_fw0(rec, 0, 20, a) && read_fw0(rec, 20, 20, b ? b : &tmp) && read_fw0(rec, 40, 20, c ? c : &tmp);
    };
    if (!f3(&d.fixcos, nullptr, nullptr)) return DVR3D_ERR_DECK;
    if (!r.more()) return DVR3D_ERR_DECK;
    if (!f3(&d.xmass[0], &d.xmass[1], &d.xmass[2])) return DVR3D_ERR_DECK;
    if (!f3(&d.xmassr[0], &d.xmassr[1], &d.xmassr[2])) return DVR3D_ERR_DECK;
    if (!f3(&d.emax1, &d.emax2, nullptr)) return DVR3D_ERR_DECK;
    if (!f3(&d.re1, &d.diss1, &d.we1)) return DVR3D_ERR_DECK;
    if (!f3(&d.re2, &d.diss2, &d.we2)) return DVR3D_ERR_DECK;
    d.have_ezero = 0;
    if (r.more() && r.rec[r.pos].find_first_not_of(" \t") != std::string::npos) {
        if (!read_fw0(r.next(), 0, 20, &d.ezero)) return DVR3D_ERR_DECK;
        d.have_ezero = 1;
    }
    *out = d;
    return DVR3D_OK;
}
