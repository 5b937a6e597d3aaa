// Host-side files of the reference's output routines, for drivers other than the Fortran main
// program (which keeps its own recrd / recrd2 / recrd3 / readin on the host arrays that
// dasha_get_state and dasha_current fill).
//
//  - Restart file mhdNNNRRR (recrd / readin, t3dsdsc.f:4814-4861): Fortran unformatted
//    sequential, two records: (ncase, nstep: INTEGER*4; time: REAL*8; nst: INTEGER*4) and the
//    whole array x(mxpr, my, mzpr, 8) of REAL*8 (mhd02.for:4; implicit real*8 (a-h,o-z), so
//    names in i-n are INTEGER*4), native byte order.  Record framing as gfortran writes it:
//    each record is one or more subrecords, each a 4-byte signed length, the data and the same
//    length again; the leading length is negative when another subrecord of the record
//    follows, the trailing one when another precedes; a subrecord holds at most 2147483639
//    bytes.
//  - 2-D mid-plane file m2dNNN.dat (recrd2, t3dsdsc.f:5116-5154) and 3-D file m3dNNN (recrd3,
//    t3dsdsc.f:5365-5402): list-directed lines "2 mx mz" (or "3 mx my mz") and "time", then the
//    node coordinates (x, z or x, y, z) as one output list, then for q = 1..11 a list-directed
//    line "q" and field q, x fastest, with the edit descriptors 5(1X,E14.5E3) (m2d) or
//    11(1X,E10.4) (m3d), a new line after every 5 or 11 numbers and at the end of each list.
//    Fields: 1 rho, 2-4 v = (rho v)/rho, 5-7 B, 8 p (totals), 9-11 the current density; m2d
//    holds the plane j = my/2 (0-based; nyh = my/2+1 in the reference).
//  - The main loop's step logs (t3dsdsc.f:157-181): ./data/stepnm, one list-directed line
//    "nstep time dt" appended before each step, and unit 20 (fort.20), one line
//    2(1X,F10.5),1X,I5 of dt, time and nstep after it.
//  - current.dat of diagn (t3dsdsc.f:1226-1232): one line per call, the mid-y-plane extrema
//    Jx max, Jx min, Jy max, Jy min, Jz max, Jz min and time in the format 7(1X,E13.4).  The
//    reference opens unit 9 on every call and never closes it, so the lines of a run follow
//    one another in the file.
#include "dasha_capi.h"
#include "fortran_format.h"
#include "fortran_records.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <thread>
#include <vector>

namespace {

using dasha::File;
using dasha::ld_ints;
using dasha::ld_real;
using dasha::ListWriter;
using dasha::fmt_f;
using dasha::fmt_i;
using dasha::write_list;
using dasha::kMaxSubrecord;
using dasha::pack_restart_header;
using dasha::unpack_restart_header;
using dasha::RecReader;
using dasha::RecWriter;

inline long hidx(long ld1, long ld2, int mz, int i, int j, int k, int m) {
    return (long)(i + 2) + ld1 * ((long)j + ld2 * ((long)(k + 2) + (long)(mz + 4) * m));
}

// value of m2d/m3d field q (0..10) at node (i,j,k) from the state and current arrays
inline double out_field(const double* x_f, const double* cur_f, long ld1, long ld2, int mz, int q, int i, int j,
                        int k) {
    if (q >= 8) return cur_f[hidx(ld1, ld2, mz, i, j, k, q - 8)];
    const double v = x_f[hidx(ld1, ld2, mz, i, j, k, q)];
    return (q >= 1 && q <= 3) ? v / x_f[hidx(ld1, ld2, mz, i, j, k, 0)] : v;
}

bool dims_ok(int mx, int my, int mz, long ld1, long ld2) {
    return mx > 0 && my > 0 && mz > 0 && ld1 >= mx + 4 && ld2 >= my;
}

}  // namespace

// Runs the body of an entry point: a host exception (allocation, thread start) becomes a
// status, as no exception may cross the C-ABI.
template <class F>
static int guarded(F body) {
    try {
        return body();
    } catch (const std::bad_alloc&) {
        return DASHA_E_NOMEM;
    } catch (...) {
        return DASHA_E_INVALID;
    }
}

extern "C" {

int dasha_restart_write(const char* path, int ncase, int nstep, double time, int nst, int mx, int my, int mz,
                        const double* x_f, long ld1, long ld2, long max_subrecord) {
    if (!path || !x_f || !dims_ok(mx, my, mz, ld1, ld2) || max_subrecord < 0) return DASHA_E_INVALID;
    return guarded([&]() -> int {
        const long maxsub = max_subrecord == 0 ? kMaxSubrecord : std::min(max_subrecord, kMaxSubrecord);
        File f(path, "wb");
        if (!f.f) return DASHA_E_INVALID;
        unsigned char hdr[20];
        pack_restart_header(hdr, ncase, nstep, time, nst);
        RecWriter w1(f.f, 20, maxsub);
        w1.put(hdr, 20);
        if (!w1.finish()) return DASHA_E_INVALID;
        const long row = mx + 4, nrow = (long)my * (mz + 4) * 8;
        RecWriter w(f.f, (long)sizeof(double) * row * nrow, maxsub);
        if (ld1 == row && ld2 == my) {
            w.put(x_f, (long)sizeof(double) * row * nrow);
        } else {
            for (int m = 0; m < 8 && w.ok; ++m)
                for (int kk = 0; kk < mz + 4 && w.ok; ++kk)
                    for (int j = 0; j < my; ++j)
                        w.put(x_f + ld1 * ((long)j + ld2 * ((long)kk + (long)(mz + 4) * m)), (long)sizeof(double) * row);
        }
        const bool ok = w.finish();
        return f.close() && ok ? DASHA_OK : DASHA_E_INVALID;
    });
}

int dasha_restart_read(const char* path, int* ncase, int* nstep, double* time, int* nst, int mx, int my, int mz,
                       double* x_f, long ld1, long ld2) {
    if (!path || !ncase || !nstep || !time || !nst || !x_f || !dims_ok(mx, my, mz, ld1, ld2)) return DASHA_E_INVALID;
    return guarded([&]() -> int {
        File f(path, "rb");
        if (!f.f) return DASHA_E_INVALID;
        unsigned char hdr[20];
        RecReader r1(f.f, 20);
        r1.get(hdr, 20);
        if (!r1.finish()) return DASHA_E_INVALID;
        const long row = mx + 4, nrow = (long)my * (mz + 4) * 8;
        RecReader r(f.f, (long)sizeof(double) * row * nrow);
        if (ld1 == row && ld2 == my) {
            r.get(x_f, (long)sizeof(double) * row * nrow);
        } else {
            for (int m = 0; m < 8 && r.ok; ++m)
                for (int kk = 0; kk < mz + 4 && r.ok; ++kk)
                    for (int j = 0; j < my; ++j)
                        r.get(x_f + ld1 * ((long)j + ld2 * ((long)kk + (long)(mz + 4) * m)), (long)sizeof(double) * row);
        }
        if (!r.finish()) return DASHA_E_INVALID;
        unpack_restart_header(hdr, ncase, nstep, time, nst);
        return DASHA_OK;
    });
}

// The restart files of an nprx x nprz MPI run of the reference (t3dsdsc.f:36-67, 4814-4861):
// rank r (mepx = r mod nprx, mepz = r / nprx) holds x(mxpr, my, mzpr, 8) with mxpr = mx/nprx + 4
// and mzpr = mz/nprz + 4; its interior columns jx = 3 .. mxpr-2 (1-based; the last rank in x
// also mxpr-1 when mod(mx, nprx) = 1) are the global columns mepx*(mxpr-4) + jx - 2, and the
// same in z.  The reference allows mod(mx, nprx) <= 1 and mod(mz, nprz) <= 1 only (T:44-47).
struct RankGrid {
    int mx, my, mz, nprx, nprz, mxpr, mzpr;
    bool ok() const {
        return nprx > 0 && nprz > 0 && nprx * nprz <= 1000 && mx % nprx <= 1 && mz % nprz <= 1 && mx / nprx >= 1 &&
               mz / nprz >= 1;
    }
    // local 0-based column range [lo, hi] of rank coordinate p holding global nodes
    void interior(int p, int npr, int mpr, int m, int* lo, int* hi) const {
        *lo = 2;
        *hi = mpr - 3 + (p == npr - 1 ? m % npr : 0);
    }
    std::string path(const char* dir, int nst, int rank) const {
        char name[16];
        std::snprintf(name, sizeof name, "mhd%03d%03d", nst, rank);
        return std::string(dir) + "/" + name;
    }
};

int dasha_restart_read_ranks(const char* dir, int nst_file, int nprx, int nprz, int* ncase, int* nstep, double* time,
                             int* nst, int mx, int my, int mz, double* x_f, long ld1, long ld2) {
    if (!dir || !ncase || !nstep || !time || !nst || !x_f || !dims_ok(mx, my, mz, ld1, ld2)) return DASHA_E_INVALID;
    RankGrid G{mx, my, mz, nprx, nprz, mx / std::max(nprx, 1) + 4, mz / std::max(nprz, 1) + 4};
    if (!G.ok() || nst_file < 0 || nst_file > 999) return DASHA_E_INVALID;
    return guarded([&]() -> int {
        const long nloc = (long)G.mxpr * my * G.mzpr * 8;
        std::vector<double> loc((size_t)nloc);
        unsigned char hdr0[20] = {0};
        for (int r = 0; r < nprx * nprz; ++r) {
            File f(G.path(dir, nst_file, r).c_str(), "rb");
            if (!f.f) return DASHA_E_INVALID;
            unsigned char hdr[20];
            RecReader r1(f.f, 20);
            r1.get(hdr, 20);
            RecReader r2(f.f, (long)sizeof(double) * nloc);
            if (r1.finish()) r2.get(loc.data(), (long)sizeof(double) * nloc);
            if (!r1.finish() || !r2.finish()) return DASHA_E_INVALID;
            if (r == 0) std::memcpy(hdr0, hdr, 20);
            else if (std::memcmp(hdr0, hdr, 20) != 0) return DASHA_E_INVALID;   // ranks of different runs
            const int px = r % nprx, pz = r / nprx;
            int xlo, xhi, zlo, zhi;
            G.interior(px, nprx, G.mxpr, mx, &xlo, &xhi);
            G.interior(pz, nprz, G.mzpr, mz, &zlo, &zhi);
            for (int m = 0; m < 8; ++m)
                for (int lz = zlo; lz <= zhi; ++lz)
                    for (int j = 0; j < my; ++j) {
                        const int gk = pz * (G.mzpr - 4) + lz - 2, gi0 = px * (G.mxpr - 4) + xlo - 2;
                        const double* src = loc.data() + xlo + (long)G.mxpr * (j + (long)my * (lz + (long)G.mzpr * m));
                        std::memcpy(x_f + hidx(ld1, ld2, mz, gi0, j, gk, m), src, sizeof(double) * (xhi - xlo + 1));
                    }
        }
        unpack_restart_header(hdr0, ncase, nstep, time, nst);
        return DASHA_OK;
    });
}

int dasha_restart_write_ranks(const char* dir, int ncase, int nstep, double time, int nst, int nprx, int nprz, int mx,
                              int my, int mz, const double* x_f, long ld1, long ld2, long max_subrecord) {
    if (!dir || !x_f || !dims_ok(mx, my, mz, ld1, ld2) || max_subrecord < 0) return DASHA_E_INVALID;
    RankGrid G{mx, my, mz, nprx, nprz, mx / std::max(nprx, 1) + 4, mz / std::max(nprz, 1) + 4};
    if (!G.ok() || nst < 0 || nst > 999) return DASHA_E_INVALID;
    return guarded([&]() -> int {
        const long maxsub = max_subrecord == 0 ? kMaxSubrecord : std::min(max_subrecord, kMaxSubrecord);
        const long nloc = (long)G.mxpr * my * G.mzpr * 8;
        std::vector<double> loc((size_t)nloc);
        unsigned char hdr[20];
        pack_restart_header(hdr, ncase, nstep, time, nst);
        for (int r = 0; r < nprx * nprz; ++r) {
            const int px = r % nprx, pz = r / nprx;
            // every local entry from the global node it stands for: x wraps (periodic), z
            // beyond the walls is zero
            for (int m = 0; m < 8; ++m)
                for (int lz = 0; lz < G.mzpr; ++lz)
                    for (int j = 0; j < my; ++j)
                        for (int lx = 0; lx < G.mxpr; ++lx) {
                            const int gk = pz * (G.mzpr - 4) + lz - 2;
                            int gi = px * (G.mxpr - 4) + lx - 2;
                            gi = ((gi % mx) + mx) % mx;
                            loc[lx + (size_t)G.mxpr * (j + (size_t)my * (lz + (size_t)G.mzpr * m))] =
                                (gk >= 0 && gk < mz) ? x_f[hidx(ld1, ld2, mz, gi, j, gk, m)] : 0.0;
                        }
            File f(G.path(dir, nst, r).c_str(), "wb");
            if (!f.f) return DASHA_E_INVALID;
            RecWriter w1(f.f, 20, maxsub);
            w1.put(hdr, 20);
            RecWriter w2(f.f, (long)sizeof(double) * nloc, maxsub);
            if (w1.finish()) w2.put(loc.data(), (long)sizeof(double) * nloc);
            if (!w1.finish() || !w2.finish() || !f.close()) return DASHA_E_INVALID;
        }
        return DASHA_OK;
    });
}

int dasha_m2d_write(const char* path, int mx, int mz, double time, const double* xc, const double* zc,
                    const double* plane) {
    if (!path || mx <= 0 || mz <= 0 || !xc || !zc || !plane) return DASHA_E_INVALID;
    return guarded([&]() -> int {
        File f(path, "w");
        if (!f.f) return DASHA_E_INVALID;
        const int hdr[3] = {2, mx, mz};
        ld_ints(f.f, hdr, 3);
        ld_real(f.f, time);
        bool ok = write_list(f.f, (long)mx + mz, 5, 14, 5, 3, [&](long n) { return n < mx ? xc[n] : zc[n - mx]; });
        const long np = (long)mx * mz;
        for (int q = 0; q < 11 && ok; ++q) {
            const int iq = q + 1;
            ld_ints(f.f, &iq, 1);
            const double* p = plane + (size_t)q * np;
            ok = write_list(f.f, np, 5, 14, 5, 3, [&](long n) { return p[n]; });
        }
        return f.close() && ok ? DASHA_OK : DASHA_E_INVALID;
    });
}

int dasha_m3d_write(const char* path, int mx, int my, int mz, double time, const double* xc, const double* yc,
                    const double* zc, const double* x_f, const double* cur_f, long ld1, long ld2) {
    if (!path || !xc || !yc || !zc || !x_f || !cur_f || !dims_ok(mx, my, mz, ld1, ld2)) return DASHA_E_INVALID;
    return guarded([&]() -> int {
        File f(path, "w");
        if (!f.f) return DASHA_E_INVALID;
        const int hdr[4] = {3, mx, my, mz};
        ld_ints(f.f, hdr, 4);
        ld_real(f.f, time);
        bool ok = write_list(f.f, (long)mx + my + mz, 11, 10, 4, 0, [&](long n) {
            return n < mx ? xc[n] : (n < (long)mx + my ? yc[n - mx] : zc[n - mx - my]);
        });
        const long mxy = (long)mx * my;
        for (int q = 0; q < 11 && ok; ++q) {
            const int iq = q + 1;
            ld_ints(f.f, &iq, 1);
            ListWriter lw(f.f, 11, 10, 4, 0);   // one plane per put: records run across planes
            for (int k = 0; k < mz && lw.ok; ++k)
                lw.put(mxy, [&](long n) { return out_field(x_f, cur_f, ld1, ld2, mz, q, (int)(n % mx), (int)(n / mx), k); });
            ok = lw.end();
        }
        return f.close() && ok ? DASHA_OK : DASHA_E_INVALID;
    });
}

int dasha_current_dat_write(const char* path, const double* diag, double time, int append) {
    if (!path || !diag) return DASHA_E_INVALID;
    return guarded([&]() -> int {
        File f(path, append ? "a" : "w");
        if (!f.f) return DASHA_E_INVALID;
        const double v[7] = {diag[3], diag[4], diag[5], diag[6], diag[7], diag[8], time};
        const bool ok = write_list(f.f, 7, 7, 13, 4, 0, [&](long n) { return v[n]; });
        return f.close() && ok ? DASHA_OK : DASHA_E_INVALID;
    });
}

int dasha_stepnm_write(const char* path, int nstep, double time, double dt) {
    if (!path) return DASHA_E_INVALID;
    return guarded([&]() -> int {
        File f(path, "a");
        if (!f.f) return DASHA_E_INVALID;
        std::fprintf(f.f, " %11d %24.16E %24.16E\n", nstep, time, dt);
        return f.close() ? DASHA_OK : DASHA_E_INVALID;
    });
}

int dasha_dtlog_write(const char* path, double dt, double time, int nstep) {
    if (!path) return DASHA_E_INVALID;
    return guarded([&]() -> int {
        File f(path, "a");
        if (!f.f) return DASHA_E_INVALID;
        char line[40];
        line[0] = ' ';
        fmt_f(line + 1, dt, 10, 5);
        line[11] = ' ';
        fmt_f(line + 12, time, 10, 5);
        line[22] = ' ';
        fmt_i(line + 23, nstep, 5);
        line[28] = '\n';
        const bool ok = std::fwrite(line, 1, 29, f.f) == 29;
        return f.close() && ok ? DASHA_OK : DASHA_E_INVALID;
    });
}

int dasha_midplane_host(int mx, int my, int mz, const double* x_f, const double* cur_f, long ld1, long ld2,
                        double* plane) {
    if (!x_f || !cur_f || !plane || !dims_ok(mx, my, mz, ld1, ld2)) return DASHA_E_INVALID;
    const int j = my / 2;
    const long np = (long)mx * mz;
    for (int q = 0; q < 11; ++q)
        for (int k = 0; k < mz; ++k)
            for (int i = 0; i < mx; ++i) plane[q * np + i + (long)mx * k] = out_field(x_f, cur_f, ld1, ld2, mz, q, i, j, k);
    return DASHA_OK;
}

}  // extern "C"
