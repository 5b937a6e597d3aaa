// Fortran unformatted sequential records as gfortran writes them (host code): each record is
// one or more subrecords, each a 4-byte signed length, the data and the same length again; the
// leading length is negative when another subrecord of the record follows, the trailing one
// when another precedes; a subrecord holds at most 2147483639 bytes.  Used for the reference's
// restart file (recrd / readin, t3dsdsc.f:4814-4861).
#pragma once

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>

namespace dasha {

constexpr long kMaxSubrecord = 2147483639L;   // gfortran's longest subrecord

// Streams one logical record of known length as subrecords of at most maxsub bytes.
struct RecWriter {
    FILE* f;
    long total, maxsub, done = 0, left_in_sub = 0, cur_open_len = 0;
    bool ok = true, first = true;
    RecWriter(FILE* f_, long total_, long maxsub_) : f(f_), total(total_), maxsub(maxsub_) {
        if (total == 0) { open_sub(); close_sub(); }
    }
    void marker(int32_t v) { ok = ok && std::fwrite(&v, 4, 1, f) == 1; }
    void open_sub() {
        cur_open_len = std::min(total - done, maxsub);
        left_in_sub = cur_open_len;
        marker(done + cur_open_len < total ? -(int32_t)cur_open_len : (int32_t)cur_open_len);
    }
    void close_sub() {
        marker(first ? (int32_t)cur_open_len : -(int32_t)cur_open_len);
        first = false;
    }
    void put(const void* data, long n) {
        const char* p = static_cast<const char*>(data);
        while (n > 0 && ok) {
            if (done >= total) { ok = false; break; }   // more data than the record holds
            if (left_in_sub == 0) open_sub();
            const long m = std::min(n, left_in_sub);
            ok = ok && std::fwrite(p, 1, (size_t)m, f) == (size_t)m;
            p += m; n -= m; done += m; left_in_sub -= m;
            if (left_in_sub == 0) close_sub();
        }
    }
    bool finish() const { return ok && done == total && left_in_sub == 0; }
};

// Reads one logical record that must hold exactly `total` bytes, subrecord by subrecord.
struct RecReader {
    FILE* f;
    long total, done = 0, left_in_sub = 0, sub_len = 0;
    bool ok = true, first = true, more = true;
    RecReader(FILE* f_, long total_) : f(f_), total(total_) {
        if (total == 0) { open_sub(); close_sub(); }
    }
    int32_t marker() {
        int32_t v = 0;
        ok = ok && std::fread(&v, 4, 1, f) == 1;
        return v;
    }
    void open_sub() {
        if (!more) { ok = false; return; }
        const int32_t h = marker();
        more = h < 0;
        sub_len = more ? -(long)h : (long)h;
        left_in_sub = sub_len;
        if (done + sub_len > total) ok = false;
    }
    void close_sub() {
        const int32_t t = marker();
        if ((first ? (long)t : -(long)t) != sub_len) ok = false;
        first = false;
    }
    void get(void* out, long n) {
        char* p = static_cast<char*>(out);
        while (n > 0 && ok) {
            while (left_in_sub == 0 && ok) {   // zero-length subrecords carry nothing
                open_sub();
                if (ok && left_in_sub == 0) close_sub();
            }
            if (!ok) break;
            const long m = std::min(n, left_in_sub);
            ok = ok && std::fread(p, 1, (size_t)m, f) == (size_t)m;
            p += m; n -= m; done += m; left_in_sub -= m;
            if (left_in_sub == 0) close_sub();
        }
    }
    bool finish() const { return ok && done == total && !more && left_in_sub == 0; }
};

// Walks the markers of one record from the current position without reading its data:
// true if they are consistent and the record holds exactly `total` bytes.  The position is
// restored either way.
inline bool scan_record(FILE* f, long total) {
    const long start = std::ftell(f);
    long done = 0;
    bool first = true, ok = start >= 0;
    for (;;) {
        int32_t h = 0, t = 0;
        if (!ok || std::fread(&h, 4, 1, f) != 1) { ok = false; break; }
        const bool more = h < 0;
        const long n = more ? -(long)h : (long)h;
        if (done + n > total || std::fseek(f, n, SEEK_CUR) != 0 || std::fread(&t, 4, 1, f) != 1 ||
            (first ? (long)t : -(long)t) != n) { ok = false; break; }
        done += n;
        first = false;
        if (!more) break;
    }
    ok = ok && done == total;
    if (start >= 0) std::fseek(f, start, SEEK_SET);
    return ok;
}

// Record 1 of the restart file: ncase, nstep (INTEGER*4), time (REAL*8), nst (INTEGER*4).
inline void pack_restart_header(unsigned char* h, int ncase, int nstep, double time, int nst) {
    const int32_t a = ncase, b = nstep, d = nst;
    std::memcpy(h, &a, 4);
    std::memcpy(h + 4, &b, 4);
    std::memcpy(h + 8, &time, 8);
    std::memcpy(h + 16, &d, 4);
}
inline void unpack_restart_header(const unsigned char* h, int* ncase, int* nstep, double* time, int* nst) {
    int32_t a, b, d;
    std::memcpy(&a, h, 4);
    std::memcpy(&b, h + 4, 4);
    std::memcpy(time, h + 8, 8);
    std::memcpy(&d, h + 16, 4);
    *ncase = a;
    *nstep = b;
    *nst = d;
}

// A FILE* closed when it leaves scope (also when an exception passes); close() reports whether
// the buffered data reached the file.
struct File {
    FILE* f = nullptr;
    File(const char* path, const char* mode) : f(std::fopen(path, mode)) {}
    File(const File&) = delete;
    File& operator=(const File&) = delete;
    ~File() { if (f) std::fclose(f); }
    bool close() {
        const bool ok = f && !std::ferror(f) && std::fclose(f) == 0;
        f = nullptr;
        return ok;
    }
};

}  // namespace dasha
