// Fortran formatted output as the reference's WRITE statements produce it (host code): E, F
// and I editing, output lists under a repeated edit descriptor, and list-directed lines.  Used
// for the reference's ASCII outputs (m2d, m3d, current.dat and the step logs).
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

namespace dasha {

// Powers of ten 1e-300 .. 1e300 as correctly rounded doubles (strtod), exact up to 1e22.
struct Pow10 {
    double p[601];
    Pow10() {
        for (int k = -300; k <= 300; ++k) p[k + 300] = std::strtod(("1e" + std::to_string(k)).c_str(), nullptr);
    }
};
inline const Pow10& pow10_table() {
    static const Pow10 t;
    return t;
}

// The d (<= 6) significant decimal digits of a > 0, correctly rounded, and the exponent e of
// a ~ 0.d1..dd x 10^e, by scaling in double: m = a * 10^(d-1-e10) lies in [10^(d-1), 10^d)
// with a relative error below 3e-16 (two roundings), so below 3e-10 in absolute terms, and
// rounding m to the nearest integer gives the exact result unless m lies within 1e-6 of a
// tie (xxx.5) or of either end of the interval, where the function declines (returns false)
// and the caller uses the exact conversion of snprintf.
inline bool fast_digits(double a, int d, char* digits, int* e) {
    if (d < 1 || d > 6 || !(a >= 1e-280 && a <= 1e280)) return false;
    static const double P[7] = {1, 10, 100, 1000, 10000, 100000, 1000000};
    int e10 = (int)std::floor(std::log10(a));
    const int sc = d - 1 - e10;
    if (sc < -300 || sc > 300) return false;
    const double m = a * pow10_table().p[sc + 300];
    const double lo = P[d - 1], hi = P[d];
    if (!(m >= lo + 1e-6 && m <= hi - 1e-6)) return false;   // exponent near a power of ten
    const double fl = std::floor(m), fr = m - fl;            // exact: m < 1e6
    if (std::fabs(fr - 0.5) < 1e-6) return false;            // near a decimal tie
    long r = (long)fl + (fr > 0.5 ? 1 : 0);
    if (r >= (long)hi) { r = (long)lo; ++e10; }              // 9..9.7 rounds up to 10..0
    for (int q = d - 1; q >= 0; --q) { digits[q] = char('0' + r % 10); r /= 10; }
    *e = e10 + 1;
    return true;
}

// Fortran Ew.d (edig = 0) or Ew.dEe output editing of v at scale factor 0, as gfortran writes it:
// [-][0].d1..dd followed by E+xx (Ew.d, |exponent| <= 99), +xxx (Ew.d, 99 < |exponent| <= 999)
// or E+ and edig digits; the optional zero before the point is written when the width has
// room; a field that does not fit is w asterisks.  Writes exactly w characters, no terminator.
inline void fmt_e(char* out, double v, int w, int d, int edig) {
    char body[64];
    const bool neg = std::signbit(v);
    if (std::isnan(v) || std::isinf(v)) {
        const char* s = std::isnan(v) ? "NaN" : (neg ? (w >= 9 ? "-Infinity" : "-Inf") : (w >= 8 ? "Infinity" : "Inf"));
        const int n = (int)std::strlen(s);
        if (n > w) { std::memset(out, '*', w); return; }
        std::memset(out, ' ', w - n);
        std::memcpy(out + w - n, s, n);
        return;
    }
    char digits[32];
    int e = 0;
    if (v == 0.0) {
        std::memset(digits, '0', d);
    } else if (!fast_digits(std::fabs(v), d, digits, &e)) {
        char s[48];
        std::snprintf(s, sizeof s, "%.*e", d - 1, std::fabs(v));   // d.dd..de+XX: d significant digits
        digits[0] = s[0];
        if (d > 1) std::memcpy(digits + 1, s + 2, d - 1);
        e = std::atoi(std::strchr(s, 'e') + 1) + 1;                 // 0.d1..dd x 10^e
    }
    const int ae = e < 0 ? -e : e;
    // exponent field: E, sign and nd digits (Ew.d with |e| <= 99, Ew.dEe), or sign and 3 digits
    int nd;
    bool with_e = true;
    if (edig == 0) {
        if (ae <= 99) nd = 2;
        else if (ae <= 999) { nd = 3; with_e = false; }
        else { std::memset(out, '*', w); return; }
    } else {
        int lim = 1;
        for (int q = 0; q < edig; ++q) lim *= 10;
        if (ae >= lim) { std::memset(out, '*', w); return; }
        nd = edig;
    }
    char ex[16];
    int nex = 0;
    if (with_e) ex[nex++] = 'E';
    ex[nex++] = e < 0 ? '-' : '+';
    for (int q = nd - 1, a = ae; q >= 0; --q, a /= 10) ex[nex + q] = char('0' + a % 10);
    nex += nd;
    const int need = (neg ? 1 : 0) + 1 + d + nex;   // without the optional zero
    if (need > w) { std::memset(out, '*', w); return; }
    int n = 0;
    if (neg) body[n++] = '-';
    if (need + 1 <= w) body[n++] = '0';
    body[n++] = '.';
    std::memcpy(body + n, digits, d);
    n += d;
    std::memcpy(body + n, ex, nex);
    n += nex;
    std::memset(out, ' ', w - n);
    std::memcpy(out + w - n, body, n);
}

// Fortran Fw.d output editing of v: correctly rounded to d decimals (snprintf), right-justified;
// the optional zero before the point is dropped only when the field would not fit otherwise;
// a field that does not fit is w asterisks.  Writes exactly w characters, no terminator.
inline void fmt_f(char* out, double v, int w, int d) {
    char s[512];
    int n = std::snprintf(s, sizeof s, "%.*f", d, v);
    const char* p = s;
    if (n > w && (std::strncmp(s, "0.", 2) == 0 || std::strncmp(s, "-0.", 3) == 0)) {
        if (s[0] == '-') { s[1] = '-'; p = s + 1; } else p = s + 1;
        --n;
    }
    if (n > w || n < 0 || !std::isfinite(v)) { std::memset(out, '*', w); return; }
    std::memset(out, ' ', w - n);
    std::memcpy(out + w - n, p, n);
}

// Fortran Iw output editing: right-justified, w asterisks when it does not fit.
inline void fmt_i(char* out, long v, int w) {
    char s[32];
    const int n = std::snprintf(s, sizeof s, "%ld", v);
    if (n > w) { std::memset(out, '*', w); return; }
    std::memset(out, ' ', w - n);
    std::memcpy(out + w - n, s, n);
}

// `nlines` full records of an output list under r(1X,Ew.d[Ee]), r = per_line, item n given by
// value(n): blocks of lines are formatted in parallel and written in order.
template <class F>
bool write_lines(FILE* f, long nlines, int per_line, int w, int d, int edig, F value) {
    const int lw = per_line * (w + 1) + 1;
    const long block = 1L << 14;   // lines per block
    const unsigned nt = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    std::vector<std::string> buf(nt);
    for (long l0 = 0; l0 < nlines; l0 += block * nt) {
        std::vector<std::thread> th;
        for (unsigned t = 0; t < nt; ++t) {
            th.emplace_back([&, t]() {
                std::string& s = buf[t];
                s.clear();
                const long a = l0 + (long)t * block, b = std::min(nlines, a + block);
                if (a >= b) return;
                s.resize((size_t)(b - a) * lw);
                char* p = &s[0];
                for (long l = a; l < b; ++l) {
                    for (long n = l * per_line; n < (l + 1) * per_line; ++n) {
                        *p++ = ' ';
                        fmt_e(p, value(n), w, d, edig);
                        p += w;
                    }
                    *p++ = '\n';
                }
            });
        }
        for (auto& x : th) x.join();
        for (unsigned t = 0; t < nt; ++t)
            if (!buf[t].empty() && std::fwrite(buf[t].data(), 1, buf[t].size(), f) != buf[t].size()) return false;
    }
    return true;
}

// An output list under r(1X,Ew.d[Ee]) written in pieces: a record (line) that a put() leaves
// open continues in the next put(), and end() closes the last one, so the text is the same
// however the items are split between calls.
struct ListWriter {
    FILE* f;
    int per_line, w, d, edig;
    int col = 0;   // items in the open record
    bool ok = true;
    ListWriter(FILE* f_, int per_line_, int w_, int d_, int edig_)
        : f(f_), per_line(per_line_), w(w_), d(d_), edig(edig_) {}
    template <class F>
    void put(long count, F value) {
        long n = 0;
        std::string s;
        auto item = [&](double v) {
            const size_t at = s.size();
            s.resize(at + 1 + w);
            s[at] = ' ';
            fmt_e(&s[at + 1], v, w, d, edig);
        };
        while (col > 0 && n < count) {   // the rest of the open record
            item(value(n++));
            if (++col == per_line) { s += '\n'; col = 0; }
        }
        if (!s.empty()) { ok = ok && std::fwrite(s.data(), 1, s.size(), f) == s.size(); s.clear(); }
        const long full = (count - n) / per_line;
        if (full > 0) {
            const long n0 = n;
            ok = ok && write_lines(f, full, per_line, w, d, edig, [&](long q) { return value(n0 + q); });
            n += full * per_line;
        }
        while (n < count) { item(value(n++)); ++col; }   // the start of the next record
        if (!s.empty()) ok = ok && std::fwrite(s.data(), 1, s.size(), f) == s.size();
    }
    bool end() {
        if (col) { ok = ok && std::fputc('\n', f) != EOF; col = 0; }
        return ok;
    }
};

// One whole output list: the items of value(0 .. count-1), the last record closed.
template <class F>
bool write_list(FILE* f, long count, int per_line, int w, int d, int edig, F value) {
    ListWriter lw(f, per_line, w, d, edig);
    lw.put(count, value);
    return lw.end();
}

// list-directed lines: integers in 12 columns, a REAL*8 as " " + 17 significant digits
inline void ld_ints(FILE* f, const int* v, int n) {
    for (int q = 0; q < n; ++q) std::fprintf(f, " %11d", v[q]);
    std::fputc('\n', f);
}
inline void ld_real(FILE* f, double v) { std::fprintf(f, " %24.16E\n", v); }

}  // namespace dasha
