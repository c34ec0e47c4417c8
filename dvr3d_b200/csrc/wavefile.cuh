// wavefile.cuh -- reader of the suite's sequential unformatted files (the wavefunction files
// of DVR3DRJZ and ROTLEV3B): records framed by a 4-byte length before and after.
#pragma once

#include <cstdint>
#include <cstring>
#include <fstream>
#include <iterator>
#include <string>
#include <utility>
#include <vector>

#include <cstdio>

#include "../../include/dvr3d_b200.h"
#include "host_setup.h"

namespace dvr3d {

struct Records {
    std::vector<unsigned char> buf;
    std::vector<std::pair<size_t, size_t>> rec;  // (offset, bytes)
    size_t next = 0;

    [[noreturn]] static void bad(const std::string &m) { throw HostError{DVR3D_ERR_ARG, m}; }

    explicit Records(const std::string &path) {
        std::ifstream f(path, std::ios::binary);
        if (!f) bad("cannot open the wavefunction file " + path);
        buf.assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
        size_t pos = 0;
        while (pos + 8 <= buf.size()) {
            int32_t n = 0, m = 0;
            std::memcpy(&n, &buf[pos], 4);
            if (n < 0 || pos + 8 + (size_t)n > buf.size()) bad("wavefunction file: broken record framing");
            std::memcpy(&m, &buf[pos + 4 + n], 4);
            if (m != n) bad("wavefunction file: record lengths before and after differ");
            rec.emplace_back(pos + 4, (size_t)n);
            pos += 8 + (size_t)n;
        }
        if (pos != buf.size()) bad("wavefunction file: trailing bytes");
    }
    bool more() const { return next < rec.size(); }
    std::pair<const unsigned char *, size_t> take() {
        if (next >= rec.size()) bad("wavefunction file: ends before the expected record");
        const auto r = rec[next++];
        return {&buf[r.first], r.second};
    }
    std::pair<const unsigned char *, size_t> at(size_t idx) const {
        if (idx >= rec.size()) bad("wavefunction file: ends before the expected record");
        return {&buf[rec[idx].first], rec[idx].second};
    }
    std::vector<int> ints(size_t want_min = 0) {
        auto r = take();
        std::vector<int> v(r.second / 4);
        std::memcpy(v.data(), r.first, v.size() * 4);
        if (v.size() < want_min) bad("wavefunction file: integer record too short");
        return v;
    }
    std::vector<double> dbls(size_t want_min = 0) {
        auto r = take();
        std::vector<double> v(r.second / 8);
        std::memcpy(v.data(), r.first, v.size() * 8);
        if (v.size() < want_min) bad("wavefunction file: real record too short");
        return v;
    }
    // the first n doubles of record idx
    const double *vec(size_t idx, size_t n) const {
        if (idx >= rec.size() || rec[idx].second < n * 8) bad("wavefunction file: vector record too short");
        return reinterpret_cast<const double *>(&buf[rec[idx].first]);
    }
};

// Appends sequential unformatted records to a file.
struct RecordWriter {
    FILE *f = nullptr;
    std::vector<unsigned char> cur;
    void put(const void *p, size_t n) {
        const size_t o = cur.size();
        cur.resize(o + n);
        if (n) std::memcpy(&cur[o], p, n);
    }
    void i4(int v) { put(&v, 4); }
    void r8(double v) { put(&v, 8); }
    void end() {
        const int32_t n = (int32_t)cur.size();
        if (std::fwrite(&n, 4, 1, f) != 1 || (n && std::fwrite(cur.data(), 1, cur.size(), f) != cur.size()) ||
            std::fwrite(&n, 4, 1, f) != 1)
            throw HostError{DVR3D_ERR_ARG, "write to an output file failed"};
        cur.clear();
    }
};

}  // namespace dvr3d
