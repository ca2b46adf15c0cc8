// fortran_io.h -- the reference's file formats as its gfortran build writes them: unformatted
// sequential records (with subrecords beyond 2 GiB) and list-directed text output.  Shared by
// the host drivers mrlbm_run (2d_mrlbm.f90's files) and mrlbm_statistics (2d_statistics.f90's).
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

namespace {

// Fortran unformatted sequential record: 4-byte length markers around the data; records
// longer than 2147483639 bytes are split into subrecords the way gfortran does (leading
// marker negative when the record continues, trailing marker negative when the subrecord
// continues a previous one).
struct FortranWriter {
    FILE* f = nullptr;
    std::vector<char> rec;
    explicit FortranWriter(const std::string& path, const char* mode = "wb") { f = std::fopen(path.c_str(), mode); }
    ~FortranWriter() { if (f) std::fclose(f); }
    template <class T> void put(const T* p, size_t n) {
        const char* c = (const char*)p;
        rec.insert(rec.end(), c, c + n * sizeof(T));
    }
    template <class T> void put1(T v) { put(&v, 1); }
    void end_record() {
        const size_t maxsub = 2147483639u;
        size_t off = 0, total = rec.size();
        bool first = true;
        do {
            const size_t len = std::min(maxsub, total - off);
            const bool more = off + len < total;
            const int32_t lead = more ? -(int32_t)len : (int32_t)len;
            const int32_t trail = first ? (int32_t)len : -(int32_t)len;
            std::fwrite(&lead, 4, 1, f);
            if (len) std::fwrite(rec.data() + off, 1, len, f);
            std::fwrite(&trail, 4, 1, f);
            off += len;
            first = false;
        } while (off < total);
        rec.clear();
    }
};

bool read_fortran_record(FILE* f, std::vector<char>& out) {
    out.clear();
    while (true) {
        int32_t lead;
        if (std::fread(&lead, 4, 1, f) != 1) return false;
        const size_t len = (size_t)std::abs(lead);
        const size_t at = out.size();
        out.resize(at + len);
        if (len && std::fread(out.data() + at, 1, len, f) != len) return false;
        int32_t trail;
        if (std::fread(&trail, 4, 1, f) != 1) return false;
        if (lead >= 0) return true;
    }
}

// list-directed output of gfortran: integers in width 12, REAL(8) as 17 significant digits
std::string ld_int(long long v) {
    char b[32];
    std::snprintf(b, sizeof b, "%12lld", v);
    return b;
}
std::string ld_real(double v) {
    char b[64];
    const double a = std::fabs(v);
    if (v == 0.0 || (a >= 0.1 && a < 1e16)) {
        // 17 significant digits: 17 decimals below 1 (0.ddd...), fewer as the integer part grows
        const int digits_before = v == 0.0 ? 1 : std::max(0, (int)std::floor(std::log10(a)) + 1);
        std::snprintf(b, sizeof b, "%25.*f     ", std::max(0, 17 - digits_before), v);
    } else {
        std::snprintf(b, sizeof b, "%26.16E", v);
    }
    return b;
}

// list-directed output of a default REAL (single precision): 9 significant digits
std::string ld_real4(float v) {
    char b[64];
    const double a = std::fabs((double)v);
    if (v == 0.0f || (a >= 0.1 && a < 1e9)) {
        const int digits_before = v == 0.0f ? 1 : std::max(0, (int)std::floor(std::log10(a)) + 1);
        std::snprintf(b, sizeof b, "%15.*f    ", std::max(0, 9 - digits_before), (double)v);
    } else {
        std::snprintf(b, sizeof b, "%15.8E", (double)v);
    }
    return b;
}

}  // namespace
