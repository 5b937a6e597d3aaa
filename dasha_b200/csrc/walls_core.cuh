// walls_core.cuh -- the reference's own bounded configuration: the dipole magnetosphere of
// initia (t3dsdsc.f:612-850) with walls on all six sides (periodx = periody = periodz = .false.,
// mhd03.for), the x-min inflow driver (bndry, T:1710-1773), the inner-sphere mask r <= rcr (every
// bndry* routine), the radial Hall coefficient (T:1398) and a 3-D equilibrium (rhoi, bxi, byi, bzi,
// pri).  FP64 throughout, on the reference's own local layout at a 1x1 process grid: arrays
// (mxpr, my, mzpr) with mxpr = mx + 4, mzpr = mz + 4, x fastest, a field stride of
// mxpr*my*mzpr (so an 8-field state is x(mxpr, my, mzpr, 8) exactly), indices written 1-based
// as in the reference: physical nodes jx = 3..mx+2, jy = 1..my, jz = 3..mz+2; interior
// x_first..x_last = 5..mx, 3..my-2, z_first..z_last = 5..mz; boundary rows 3, 4 / mx+1, mx+2,
// 1, 2 / my-1, my and 3, 4 / mz+1, mz+2.
//
// Every routine is a sequence of loops over index boxes; each loop body is a per-node lambda
// run by an executor (`Exec::run(box, f)`; the GPU executor in walls.cu launches one thread per
// node).  The loops and their order are the reference's, so that the boundary rows, the masked
// nodes and the corners take the same values; within a loop no node reads what another node of
// the same loop writes, except where noted.  Arithmetic follows the reference's expressions term
// by term, with its single-precision constants (REAL*4 literals such as 0.15 or 1.1) as the
// float values they are.
#pragma once
#include <cmath>
#include <vector>

#if !defined(__CUDACC__)
#define __host__
#define __device__
#endif
#define WHD __host__ __device__

namespace dasha {
namespace walls {

struct Box { int x0, x1, y0, y1, z0, z1; };   // inclusive, 1-based

struct Dims {
    int mx, my, mz, mxpr, mzpr;
    long sy, sz, n;                            // strides (1, mxpr, mxpr*my) and field size
    int x_first, x_last, z_first, z_last, xfirst, xlast, zfirst, zlast;
    WHD long at(int jx, int jy, int jz) const { return (long)(jx - 1) + sy * (jy - 1) + sz * (jz - 1); }
};

// 1-D tables, indexed 1-based like the reference's arrays (entry 0 unused)
struct Tables {
    const double *xx, *yy, *zz, *dx, *dy, *dz;
    const double *ax1, *bx1, *cx1, *dx1, *ay1, *by1, *cy1, *dy1, *az1, *bz1, *cz1, *dz1;
    const double *ax2, *bx2, *cx2, *dx2, *ay2, *by2, *cy2, *dy2, *az2, *bz2, *cz2, *dz2;
    const double *axp, *bxp, *cxp;
};

struct Par {
    double gamma, eta, mu, drho, dp, cfl, rcr, chall;
    int hall, viscos, diffu;
    int uyzlimiter;
};

// device arrays of one context (padded layout); 8-field arrays hold field m at m*n
struct Arr {
    double *x, *xm, *xfold, *xdif;                 // 8 fields each
    double *cur, *efld, *xdh, *xresd;              // 3 fields each
    double *w, *fs, *gs, *hs, *u, *v;              // work fields
    double *rhoi, *bxi, *byi, *bzi, *pri, *rr0, *rr1;
    unsigned long long* dtbits;                    // setdt minimum (bits of a positive double)
};

WHD inline double d1fc(double fm2, double fm, double f0, double fp, double fp2, double a, double b, double c, double d) {
    return a * (fp - f0) + b * (f0 - fm) + c * (fp2 - f0) + d * (f0 - fm2);
}
WHD inline double difc(double fm, double f0, double fp, double xm1, double x0, double xp1) {
    return 2. * ((fp - f0) * (xp1 - x0) - (f0 - fm) * (x0 - xm1)) / (xp1 - xm1);
}
// REAL*4 constants of the reference, widened as Fortran widens them
WHD inline double real4(float v) { return (double)v; }

// ---- derivative helpers at node (jx, jy, jz) of field f ----
struct Deriv {
    Dims d;
    Tables t;
    WHD double Dx(const double* f, int jx, int jy, int jz) const {
        const long c = d.at(jx, jy, jz);
        return d1fc(f[c - 2], f[c - 1], f[c], f[c + 1], f[c + 2], t.ax1[jx], t.bx1[jx], t.cx1[jx], t.dx1[jx]);
    }
    WHD double Dy(const double* f, int jx, int jy, int jz) const {
        const long c = d.at(jx, jy, jz), s = d.sy;
        return d1fc(f[c - 2 * s], f[c - s], f[c], f[c + s], f[c + 2 * s], t.ay1[jy], t.by1[jy], t.cy1[jy], t.dy1[jy]);
    }
    WHD double Dz(const double* f, int jx, int jy, int jz) const {
        const long c = d.at(jx, jy, jz), s = d.sz;
        return d1fc(f[c - 2 * s], f[c - s], f[c], f[c + s], f[c + 2 * s], t.az1[jz], t.bz1[jz], t.cz1[jz], t.dz1[jz]);
    }
    WHD double L2(const double* f, int jx, int jy, int jz) const {   // d2fc x + y + z
        const long c = d.at(jx, jy, jz), sy = d.sy, sz = d.sz;
        return d1fc(f[c - 2], f[c - 1], f[c], f[c + 1], f[c + 2], t.ax2[jx], t.bx2[jx], t.cx2[jx], t.dx2[jx]) +
               d1fc(f[c - 2 * sy], f[c - sy], f[c], f[c + sy], f[c + 2 * sy], t.ay2[jy], t.by2[jy], t.cy2[jy], t.dy2[jy]) +
               d1fc(f[c - 2 * sz], f[c - sz], f[c], f[c + sz], f[c + 2 * sz], t.az2[jz], t.bz2[jz], t.cz2[jz], t.dz2[jz]);
    }
    // the sum of the three difc terms of a smoothing pass (avrg* routines, e.g. T:5643-5648)
    WHD double difc3(const double* f, int jx, int jy, int jz) const {
        const long c = d.at(jx, jy, jz), sy = d.sy, sz = d.sz;
        return difc(f[c - 1], f[c], f[c + 1], t.xx[jx - 1], t.xx[jx], t.xx[jx + 1]) +
               difc(f[c - sy], f[c], f[c + sy], t.yy[jy - 1], t.yy[jy], t.yy[jy + 1]) +
               difc(f[c - sz], f[c], f[c + sz], t.zz[jz - 1], t.zz[jz], t.zz[jz + 1]);
    }
    // the radial smoothing coefficient (avrg, avrgtt, avrgE, avrgc: T:5659-5661 and alike)
    WHD double coef_r(int jx, int jy, int jz) const {
        const double r = sqrt(t.xx[jx] * t.xx[jx] + t.yy[jy] * t.yy[jy] + t.zz[jz] * t.zz[jz]);
        return 1.0 / 32.0 + 0.046875 * (1 + tanh((r - 3.) / 3.));
    }
    // the x profile of the B fields in avrg / avrgtt (T:5636-5642): coef_avrg (1 - tanh((x+3)/8))
    WHD double coef_b(int jx) const { return (1.0 / 32.0) * (1 - tanh((t.xx[jx] + 3) / 8.)); }
};

// Smoothing coefficient kinds: RADIAL (coef_r * sum), BX (coef_b * sum), EIGHTH (1/8 * sum)
enum SmoothKind { SM_RADIAL = 0, SM_BX = 1, SM_EIGHTH = 2 };
// Boundary routine kinds: bndryc, bndryh, bndryE (3 fields, extrapolated x-min rows, y and z rows
// over all x), bndrytt (8 fields, extrapolated x-min rows, y and z rows from x_first), bndry (8
// fields, x-min inflow driver)
enum RowKind { ROWS_C = 0, ROWS_H = 1, ROWS_E = 2, ROWS_TT = 3, ROWS_XDIF = 4 };

template <class Exec>
struct Core {
    Exec& ex;
    Dims d;
    Tables t;
    Par p;
    Arr a;

    Deriv D() const { return Deriv{d, t}; }
    Box physical() const { return {d.x_first - 2, d.x_last + 2, 1, d.my, d.z_first - 2, d.z_last + 2}; }
    Box interior() const { return {d.x_first, d.x_last, 3, d.my - 2, d.z_first, d.z_last}; }

    // ---- one Jacobi smoothing pass of field f (w = f + coef * sum difc; f = w on the interior) ----
    void smooth(double* f, int kind) {
        const Deriv dv = D();
        double* w = a.w;
        const Dims dd = d;
        ex.run(interior(), [=] WHD(int jx, int jy, int jz) {
            const long c = dd.at(jx, jy, jz);
            const double s = dv.difc3(f, jx, jy, jz);
            if (kind == SM_RADIAL) w[c] = f[c] + dv.coef_r(jx, jy, jz) * s;
            else if (kind == SM_BX) w[c] = f[c] + dv.coef_b(jx) * s;
            else w[c] = f[c] + (1.0 / 8.0) * s;
        });
        ex.run(interior(), [=] WHD(int jx, int jy, int jz) {
            const long c = dd.at(jx, jy, jz);
            f[c] = w[c];
        });
    }

    // ---- the boundary routines: mask, x rows, y rows, z rows (bndry*, T:1677-3027) ----
    // base: first field of the array; nf fields; for ROWS_XDIF also t, ddt, km (the driver)
    void rows(int kind, double* base, int nf, double tt = 0., double ddt = 0., int km = 1) {
        const Dims dd = d;
        const Tables tb = t;
        const Par pp = p;
        const Arr aa = a;
        const long n = d.n;
        const double* rr1 = a.rr1;
        // mask: inside the sphere r <= rcr the field is 0
        ex.run(physical(), [=] WHD(int jx, int jy, int jz) {
            const long c = dd.at(jx, jy, jz);
            if (rr1[c] <= pp.rcr)
                for (int m = 0; m < nf; ++m) base[m * n + c] = 0.;
        });
        // x rows, per (jy, jz): the x-min rows (extrapolated or driven), then the x-max rows
        const Box xr{3, 3, 1, d.my, d.z_first - 2, d.z_last + 2};
        ex.run(xr, [=] WHD(int, int jy, int jz) {
            const long r3 = dd.at(3, jy, jz), r4 = dd.at(4, jy, jz);
            if (kind != ROWS_XDIF) {
                // third-order extrapolation with the one-sided weights axp, bxp, cxp (T:505-517)
                for (int m = 0; m < nf; ++m) {
                    double* f = base + m * n;
                    f[r4] = (tb.axp[4] * f[r4 + 1] + tb.bxp[4] * f[r4 + 2] + tb.cxp[4] * f[r4 + 3]) /
                            (tb.axp[4] + tb.bxp[4] + tb.cxp[4]);
                    f[r3] = (tb.axp[3] * f[r3 + 1] + tb.bxp[3] * f[r3 + 2] + tb.cxp[3] * f[r3 + 3]) /
                            (tb.axp[3] + tb.bxp[3] + tb.cxp[3]);
                }
            } else {
                // the inflow driver (T:1710-1773): the state of rows 4 and 3 is set to the
                // equilibrium plus a time-dependent density / velocity / pressure pulse, and their
                // rates to (state - start of the step) / (ddt + 1e-9).  rhoi(4,jz,jz) and
                // rhoi(3,jz,jz) index y by jz as the reference does (its defect D3), read at the same
                // linear position of the array.
                // (products in the reference's left-to-right order)
                const double zz = tb.zz[jz], yy = tb.yy[jy];
                const double at = tanh((tt - 9.) / 1.) - tanh((tt - 39.) / 1.5);
                const double bz6 = tanh((zz + real4(0.6f)) / real4(0.15f)) - tanh((zz - real4(0.6f)) / real4(0.15f));
                const double by4 = tanh((yy + real4(0.4f)) / real4(0.15f)) - tanh((yy - real4(0.4f)) / real4(0.15f));
                const double bz2 = tanh((zz + real4(0.2f)) / real4(0.15f)) - tanh((zz - real4(0.2f)) / real4(0.15f));
                const double by3 = tanh((yy + real4(0.3f)) / real4(0.15f)) - tanh((yy - real4(0.3f)) / real4(0.15f));
                // B pulse times the file field bxinfc, byinfc, bzinfc, which is 0 without the fcinp/
                // files (mxdatfc = .false.)
                const double bpulse = 0. * real4(0.0017f) * sqrt(tt * tt * tt * real4(7.25f) * real4(7.25f) * real4(7.25f)) /
                                      (exp(tt * real4(7.25f) * real4(0.0069f)) + 1.);
                double* x = aa.x;
                for (int row = 4; row >= 3; --row) {
                    const long c = row == 4 ? r4 : r3;
                    const long cd3 = dd.at(row, jz, jz);   // rhoi(row, jz, jz)
                    x[c] = aa.rhoi[cd3] + 0.5 * at * 0.5 * bz6 * 0.5 * by4;
                    x[n + c] = real4(0.8f) * x[c] * 0.5 * at * 0.5 * bz2 * 0.5 * by3;
                    x[2 * n + c] = 0.;
                    x[3 * n + c] = 0.;
                    x[4 * n + c] = aa.bxi[c] + bpulse;
                    x[5 * n + c] = aa.byi[c] + bpulse;
                    x[6 * n + c] = aa.bzi[c] + bpulse;
                    x[7 * n + c] = aa.pri[c] + (double)(0.2f * 0.5f) * at * 0.5 * bz6 * 0.5 * by4;
                }
                const double* ref = km == 1 ? aa.xfold : aa.xm;
                for (int m = 0; m < 8; ++m) {
                    base[m * n + r3] = (aa.x[m * n + r3] - ref[m * n + r3]) / (ddt + 1.e-9);
                    base[m * n + r4] = (aa.x[m * n + r4] - ref[m * n + r4]) / (ddt + 1.e-9);
                }
            }
            const long e0 = dd.at(dd.xlast, jy, jz);
            for (int m = 0; m < nf; ++m) {
                double* f = base + m * n;
                f[e0] = 0.;
                f[e0 - 1] = 0.5 * f[e0 - 2];
            }
        });
        // y rows over x
        const int yx0 = kind == ROWS_TT ? d.x_first : d.x_first - 2;
        ex.run({yx0, d.x_last + 2, 1, 1, d.z_first - 2, d.z_last + 2}, [=] WHD(int jx, int, int jz) {
            const long c1 = dd.at(jx, 1, jz), cm = dd.at(jx, dd.my, jz), sy = dd.sy;
            for (int m = 0; m < nf; ++m) {
                double* f = base + m * n;
                f[c1] = 0.;
                f[c1 + sy] = 0.5 * f[c1 + 2 * sy];
                f[cm] = 0.;
                f[cm - sy] = 0.5 * f[cm - 2 * sy];
            }
        });
        // z rows over x and y
        ex.run({yx0, d.x_last + 2, 1, d.my, 3, 3}, [=] WHD(int jx, int jy, int) {
            const long c3 = dd.at(jx, jy, 3), cl = dd.at(jx, jy, dd.zlast), sz = dd.sz;
            for (int m = 0; m < nf; ++m) {
                double* f = base + m * n;
                f[c3] = 0.;
                f[c3 + sz] = 0.5 * f[c3 + 2 * sz];
                f[cl] = 0.;
                f[cl - sz] = 0.5 * f[cl - 2 * sz];
            }
        });
        // the uy/uz limiter of bndry and bndrytt (T:1928-1975, 2231-2278): on the two wall rows
        // at each z end the z momentum, on the two rows at each y end the y momentum, may only
        // point into the domain
        if (p.uyzlimiter && (kind == ROWS_XDIF || kind == ROWS_TT)) {
            double* mz3 = base + 3 * n;
            ex.run({d.x_first, d.x_last + 2, 1, d.my, 3, 4}, [=] WHD(int jx, int jy, int jz) {
                const long c = dd.at(jx, jy, jz);
                if (mz3[c] >= 0.) mz3[c] = 0.;
            });
            ex.run({d.x_first, d.x_last + 2, 1, d.my, d.zlast - 1, d.zlast}, [=] WHD(int jx, int jy, int jz) {
                const long c = dd.at(jx, jy, jz);
                if (mz3[c] <= 0.) mz3[c] = 0.;
            });
            double* my2 = base + 2 * n;
            ex.run({d.x_first, d.x_last + 2, 1, 2, d.z_first - 2, d.z_last + 2}, [=] WHD(int jx, int jy, int jz) {
                const long c = dd.at(jx, jy, jz);
                if (my2[c] >= 0.) my2[c] = 0.;
            });
            ex.run({d.x_first, d.x_last + 2, d.my - 1, d.my, d.z_first - 2, d.z_last + 2}, [=] WHD(int jx, int jy, int jz) {
                const long c = dd.at(jx, jy, jz);
                if (my2[c] <= 0.) my2[c] = 0.;
            });
        }
    }

    // ---- current (T:2452-2500): J = curl(B - B0), bndryc, avrgc(1,3,4) ----
    void current() {
        const Dims dd = d;
        const Deriv dv = D();
        const Arr aa = a;
        const long n = d.n;
        ex.run(physical(), [=] WHD(int jx, int jy, int jz) {
            const long c = dd.at(jx, jy, jz);
            aa.u[c] = aa.x[4 * n + c] - aa.bxi[c];
            aa.v[c] = aa.x[5 * n + c] - aa.byi[c];
            aa.w[c] = aa.x[6 * n + c] - aa.bzi[c];
        });
        ex.run(interior(), [=] WHD(int jx, int jy, int jz) {
            const long c = dd.at(jx, jy, jz);
            aa.cur[c] = dv.Dy(aa.w, jx, jy, jz) - dv.Dz(aa.v, jx, jy, jz);
            aa.cur[n + c] = dv.Dz(aa.u, jx, jy, jz) - dv.Dx(aa.w, jx, jy, jz);
            aa.cur[2 * n + c] = dv.Dx(aa.v, jx, jy, jz) - dv.Dy(aa.u, jx, jy, jz);
        });
        rows(ROWS_C, a.cur, 3);
        for (int k = 0; k < 4; ++k) {
            for (int m = 0; m < 3; ++m) smooth(a.cur + m * n, SM_RADIAL);
            rows(ROWS_C, a.cur, 3);
        }
    }

    // ---- right (T:1297-1673) with totalE = .true.: xdif = dx/dt of the state x ----
    void right(double tt, double ddt, int km) {
        const Dims dd = d;
        const Deriv dv = D();
        const Arr aa = a;
        const Par pp = p;
        const long n = d.n;
        current();
        // continuity and momentum: -div of the fluxes (flux, T:2286-2347)
        for (int m = 0; m < 4; ++m) {
            ex.run(physical(), [=] WHD(int jx, int jy, int jz) {
                const long c = dd.at(jx, jy, jz);
                const double* x = aa.x;
                const double x1 = x[c], x2 = x[n + c], x3 = x[2 * n + c], x4 = x[3 * n + c], dp = x[7 * n + c] - aa.pri[c];
                if (m == 0) { aa.fs[c] = x2; aa.gs[c] = x3; aa.hs[c] = x4; }
                else if (m == 1) { aa.fs[c] = x2 * x2 / x1 + dp; aa.gs[c] = x2 * x3 / x1; aa.hs[c] = x2 * x4 / x1; }
                else if (m == 2) { aa.fs[c] = x2 * x3 / x1; aa.gs[c] = x3 * x3 / x1 + dp; aa.hs[c] = x4 * x3 / x1; }
                else { aa.fs[c] = x2 * x4 / x1; aa.gs[c] = x3 * x4 / x1; aa.hs[c] = x4 * x4 / x1 + dp; }
            });
            ex.run(interior(), [=] WHD(int jx, int jy, int jz) {
                const long c = dd.at(jx, jy, jz);
                aa.xdif[m * n + c] = -dv.Dx(aa.fs, jx, jy, jz) - dv.Dy(aa.gs, jx, jy, jz) - dv.Dz(aa.hs, jx, jy, jz);
            });
        }
        // every node: velocity, J x B - xresd, E = (-v x B) + eta J (T:1348-1373)
        ex.run(physical(), [=] WHD(int jx, int jy, int jz) {
            const long c = dd.at(jx, jy, jz);
            const double* x = aa.x;
            double* xd = aa.xdif;
            const double* cu = aa.cur;
            aa.fs[c] = x[n + c] / x[c];
            aa.gs[c] = x[2 * n + c] / x[c];
            aa.hs[c] = x[3 * n + c] / x[c];
            xd[n + c] = xd[n + c] - aa.xresd[c] + cu[n + c] * x[6 * n + c] - cu[2 * n + c] * x[5 * n + c];
            xd[2 * n + c] = xd[2 * n + c] - aa.xresd[n + c] + cu[2 * n + c] * x[4 * n + c] - cu[c] * x[6 * n + c];
            xd[3 * n + c] = xd[3 * n + c] - aa.xresd[2 * n + c] + cu[c] * x[5 * n + c] - cu[n + c] * x[4 * n + c];
            aa.efld[c] = (-x[2 * n + c] * x[6 * n + c] + x[3 * n + c] * x[5 * n + c]) / x[c] + pp.eta * cu[c];
            aa.efld[n + c] = (-x[3 * n + c] * x[4 * n + c] + x[n + c] * x[6 * n + c]) / x[c] + pp.eta * cu[n + c];
            aa.efld[2 * n + c] = (-x[n + c] * x[5 * n + c] + x[2 * n + c] * x[4 * n + c]) / x[c] + pp.eta * cu[2 * n + c];
        });
        for (int k = 0; k < 4; ++k) {                               // avrgE(t, 1, 3, 4)
            for (int m = 0; m < 3; ++m) smooth(a.efld + m * n, SM_RADIAL);
            rows(ROWS_E, a.efld, 3);
        }
        if (p.hall) {
            // cht = 0.5 chall (tanh((r0 - 1.1)/8) - tanh((r0 - 2)/10)) (T:1396-1399); xdh (T:1404-1420)
            ex.run(interior(), [=] WHD(int jx, int jy, int jz) {
                const long c = dd.at(jx, jy, jz);
                const double* x = aa.x;
                const double* cu = aa.cur;
                const double r0 = aa.rr0[c];
                const double cht = 0.5 * pp.chall * (tanh((r0 - real4(1.1f)) / 8.) - tanh((r0 - 2.) / 10.));
                const double* p8 = x + 7 * n;
                aa.xdh[c] = cht * (cu[n + c] * x[6 * n + c] - cu[2 * n + c] * x[5 * n + c] - dv.Dx(p8, jx, jy, jz)) / x[c];
                aa.xdh[n + c] = cht * (cu[2 * n + c] * x[4 * n + c] - cu[c] * x[6 * n + c] - dv.Dy(p8, jx, jy, jz)) / x[c];
                aa.xdh[2 * n + c] = cht * (cu[c] * x[5 * n + c] - cu[n + c] * x[4 * n + c] - dv.Dz(p8, jx, jy, jz)) / x[c];
            });
            rows(ROWS_H, a.xdh, 3);
            for (int k = 0; k < 5; ++k) {                           // avrgh(1, 3, 5)
                for (int m = 0; m < 3; ++m) smooth(a.xdh + m * n, SM_EIGHTH);
                rows(ROWS_H, a.xdh, 3);
            }
            ex.run(physical(), [=] WHD(int jx, int jy, int jz) {
                const long c = dd.at(jx, jy, jz);
                for (int m = 0; m < 3; ++m) aa.efld[m * n + c] = aa.efld[m * n + c] + aa.xdh[m * n + c];
            });
        }
        // induction -curl E and the pressure equation (T:1434-1566)
        ex.run(interior(), [=] WHD(int jx, int jy, int jz) {
            const long c = dd.at(jx, jy, jz);
            const double* e = aa.efld;
            const double* x = aa.x;
            double* xd = aa.xdif;
            const double* cu = aa.cur;
            xd[4 * n + c] = -dv.Dy(e + 2 * n, jx, jy, jz) + dv.Dz(e + n, jx, jy, jz);
            xd[5 * n + c] = -dv.Dz(e, jx, jy, jz) + dv.Dx(e + 2 * n, jx, jy, jz);
            xd[6 * n + c] = -dv.Dx(e + n, jx, jy, jz) + dv.Dy(e, jx, jy, jz);
            const double* p8 = x + 7 * n;
            xd[7 * n + c] = -dv.Dx(p8, jx, jy, jz) * aa.fs[c] - dv.Dy(p8, jx, jy, jz) * aa.gs[c] -
                            dv.Dz(p8, jx, jy, jz) * aa.hs[c] +
                            (-dv.Dx(aa.fs, jx, jy, jz) - dv.Dy(aa.gs, jx, jy, jz) - dv.Dz(aa.hs, jx, jy, jz)) *
                                pp.gamma * x[7 * n + c] +
                            (pp.gamma - 1.) * pp.eta * (cu[c] * cu[c] + cu[n + c] * cu[n + c] + cu[2 * n + c] * cu[2 * n + c]);
        });
        // viscosity and diffusion (T:1585-1663); with a zero coefficient the reference adds zero
        if (p.viscos && p.mu != 0.) {
            ex.run(interior(), [=] WHD(int jx, int jy, int jz) {
                const long c = dd.at(jx, jy, jz);
                double* xd = aa.xdif;
                const double af = dv.L2(aa.fs, jx, jy, jz), ag = dv.L2(aa.gs, jx, jy, jz), ah = dv.L2(aa.hs, jx, jy, jz);
                xd[n + c] = xd[n + c] + pp.mu * af;
                xd[2 * n + c] = xd[2 * n + c] + pp.mu * ag;
                xd[3 * n + c] = xd[3 * n + c] + pp.mu * ah;
                xd[7 * n + c] = xd[7 * n + c] + pp.mu * (aa.fs[c] * af + aa.gs[c] * ag + aa.hs[c] * ah);
            });
        }
        if (p.diffu && (p.drho != 0. || p.dp != 0.)) {
            ex.run(interior(), [=] WHD(int jx, int jy, int jz) {
                const long c = dd.at(jx, jy, jz);
                double* xd = aa.xdif;
                xd[c] = xd[c] + pp.drho * dv.L2(aa.x, jx, jy, jz);
                xd[7 * n + c] = xd[7 * n + c] + pp.dp * dv.L2(aa.x + 7 * n, jx, jy, jz);
            });
        }
        rows(ROWS_XDIF, a.xdif, 8, tt, ddt, km);
        if (tt != 0.) {                                              // avrg(t, ddt, km, 1, 8, 0, 2)
            for (int k = 0; k < 2; ++k) {
                for (int m = 0; m < 8; ++m) smooth(a.xdif + m * n, m >= 4 && m <= 6 ? SM_BX : SM_RADIAL);
                rows(ROWS_XDIF, a.xdif, 8, tt, ddt, km);
            }
        }
    }

    // ---- stepon (T:1063-1172): RK4 registers xfold, xm, x; then avrgtt on x - eq ----
    void stepon(double time, double dt) {
        const Dims dd = d;
        const Arr aa = a;
        const long n = d.n;
        ex.run(physical(), [=] WHD(int jx, int jy, int jz) {
            const long c = dd.at(jx, jy, jz);
            for (int m = 0; m < 8; ++m) aa.xfold[m * n + c] = aa.x[m * n + c];
        });
        const double tts[4] = {time + dt / 2, time + dt / 2, time + dt, time + dt};
        const double ddts[4] = {dt / 2., dt / 2., dt, dt / 6.};
        for (int s = 0; s < 4; ++s) {
            right(tts[s], ddts[s], s == 3 ? 2 : 1);
            ex.run(physical(), [=] WHD(int jx, int jy, int jz) {
                const long c = dd.at(jx, jy, jz);
                for (int m = 0; m < 8; ++m) {
                    const long q = m * n + c;
                    const double k = aa.xdif[q];
                    if (s == 0) { aa.xm[q] = aa.xfold[q] + k * dt / 6.; aa.x[q] = aa.xfold[q] + k * dt / 2.; }
                    else if (s == 1) { aa.xm[q] = aa.xm[q] + k * dt / 3.; aa.x[q] = aa.xfold[q] + k * dt / 2.; }
                    else if (s == 2) { aa.xm[q] = aa.xm[q] + k * dt / 3.; aa.x[q] = aa.xfold[q] + k * dt; }
                    else aa.x[q] = aa.xm[q] + k * dt / 6.;
                }
            });
        }
        const double* eq[8] = {a.rhoi, nullptr, nullptr, nullptr, a.bxi, a.byi, a.bzi, a.pri};
        ex.run(physical(), [=] WHD(int jx, int jy, int jz) {
            const long c = dd.at(jx, jy, jz);
            for (int m = 0; m < 8; ++m) aa.xm[m * n + c] = eq[m] ? aa.x[m * n + c] - eq[m][c] : aa.x[m * n + c];
        });
        const double tt = time + dt;
        for (int k = 0; k < 2; ++k) {                                // avrgtt(tt, 1, 8, 0, 2)
            for (int m = 0; m < 8; ++m) smooth(a.xm + m * n, m >= 4 && m <= 6 ? SM_BX : SM_RADIAL);
            rows(ROWS_TT, a.xm, 8, tt);
        }
        ex.run(physical(), [=] WHD(int jx, int jy, int jz) {
            const long c = dd.at(jx, jy, jz);
            for (int m = 0; m < 8; ++m) aa.x[m * n + c] = eq[m] ? aa.xm[m * n + c] + eq[m][c] : aa.xm[m * n + c];
        });
    }

    // ---- setdt (T:4694-4810): min over the cells with r >= 1 of the region zfirst..z_last,
    // 1..my-1, xfirst..x_last; one atomicMin on the bits of the positive double ----
    void setdt_launch() {
        const Dims dd = d;
        const Tables tb = t;
        const Arr aa = a;
        const Par pp = p;
        const long n = d.n;
        ex.run({d.xfirst, d.x_last, 1, d.my - 1, d.zfirst, d.z_last}, [=] WHD(int jx, int jy, int jz) {
            const long c = dd.at(jx, jy, jz);
            if (!(aa.rr1[c] >= 1.)) return;
            const double* x = aa.x;
            const double vx = x[n + c] / x[c], vy = x[2 * n + c] / x[c], vz = x[3 * n + c] / x[c];
            const double va2 = (x[4 * n + c] * x[4 * n + c] + x[5 * n + c] * x[5 * n + c] + x[6 * n + c] * x[6 * n + c]) / x[c];
            const double cs2 = pp.gamma * x[7 * n + c] / x[c];
            const double vpx = fabs(vx) + sqrt(fabs(va2 + cs2));
            const double vpy = fabs(vy) + sqrt(fabs(va2 + cs2));
            const double vpz = fabs(vz) + sqrt(fabs(va2 + cs2));
            const double vis = pp.eta + pp.mu;
            const double dtx = fabs(tb.dx[jx]) / (vpx / pp.cfl + vis / tb.dx[jx] / 2.);
            const double dty = fabs(tb.dy[jy]) / (vpy / pp.cfl + vis / tb.dy[jy] / 2.);
            const double dtz = fabs(tb.dz[jz]) / (vpz / pp.cfl + vis / tb.dz[jz] / 2.);
            const double dt1 = dtx < dty ? dtx : dty;
            const double dt2 = dtz < dt1 ? dtz : dt1;
            Exec::atomic_min_bits(aa.dtbits, dt2);
        });
    }
};


// ---- host set-up, shared by the device engine (walls.cu) and host builds of this core ----

// index ranges of a 1x1 process grid (t3dsdsc.f:60-81)
inline Dims make_dims(int mx, int my, int mz) {
    Dims d{};
    d.mx = mx; d.my = my; d.mz = mz; d.mxpr = mx + 4; d.mzpr = mz + 4;
    d.sy = d.mxpr; d.sz = (long)d.mxpr * my; d.n = d.sz * d.mzpr;
    d.x_first = 5; d.x_last = mx; d.z_first = 5; d.z_last = mz;
    d.xfirst = 3; d.xlast = mx + 2; d.zfirst = 3; d.zlast = mz + 2;
    return d;
}

// x**k as the reference's translation evaluates integer powers: repeated multiplication
inline double ipow2(double a) { return a * a; }
inline double ipow3(double a) { return a * a * a; }
inline double ipow4(double a) { const double b = a * a; return b * b; }

// The 1-D tables of input on the padded index (entry 0 unused), in the order of the members of
// Tables: xx yy zz dx dy dz; the first-derivative weights a b c d of x, y, z (T:439-504); the
// second-derivative weights (T:336-364); the one-sided weights axp bxp cxp toward +x
// (T:505-517).  Spacings are forward differences, the last one repeated.
constexpr int NTAB = 6 + 12 + 12 + 3;
inline std::vector<std::vector<double>> make_tables(const Dims& d, const double* xc, const double* yc,
                                                    const double* zc) {
    const int mx = d.mx, my = d.my, mz = d.mz;
    const int L[3] = {d.mxpr + 1, my + 1, d.mzpr + 1};
    std::vector<double> xx(L[0], 0.), yy(L[1], 0.), zz(L[2], 0.), dx(L[0], 0.), dy(L[1], 0.), dz(L[2], 0.);
    auto fwd = [](const double* c, int nn, int i) { return i + 1 < nn ? c[i + 1] - c[i] : c[i] - c[i - 1]; };
    for (int i = 0; i < mx; ++i) { xx[i + 3] = xc[i]; dx[i + 3] = fwd(xc, mx, i); }
    for (int j = 0; j < my; ++j) { yy[j + 1] = yc[j]; dy[j + 1] = fwd(yc, my, j); }
    for (int k = 0; k < mz; ++k) { zz[k + 3] = zc[k]; dz[k + 3] = fwd(zc, mz, k); }
    std::vector<double> c1[3][4], c2[3][4], cp[3];
    const std::vector<double>* crd[3] = {&xx, &yy, &zz};
    const int lo[3] = {d.x_first, 3, d.z_first}, hi[3] = {d.x_last, my - 2, d.z_last};
    for (int ax = 0; ax < 3; ++ax) {
        for (int q = 0; q < 4; ++q) { c1[ax][q].assign(L[ax], 0.); c2[ax][q].assign(L[ax], 0.); }
        const std::vector<double>& c = *crd[ax];
        for (int j = lo[ax]; j <= hi[ax]; ++j) {
            const double dxp1 = c[j + 1] - c[j], dxm1 = c[j] - c[j - 1], dxp2 = c[j + 2] - c[j], dxm2 = c[j] - c[j - 2];
            {   // second derivative (T:336-364)
                const double f1 = ipow2(dxp1) + dxp1 * dxm2, f2 = ipow3(dxp1) - dxp1 * ipow2(dxm2),
                             f3 = ipow4(dxp1) + dxp1 * ipow3(dxm2);
                const double g1 = -ipow2(dxm1) + dxm1 * dxm2, g2 = ipow3(dxm1) - dxm1 * ipow2(dxm2),
                             g3 = -ipow4(dxm1) + dxm1 * ipow3(dxm2);
                const double h1 = ipow2(dxp2) + dxp2 * dxm2, h2 = ipow3(dxp2) - dxp2 * ipow2(dxm2),
                             h3 = ipow4(dxp2) + dxp2 * ipow3(dxm2);
                const double ca = (f1 * h3 - f3 * h1) * (g2 * h3 - g3 * h2) - (g1 * h3 - g3 * h1) * (f2 * h3 - f3 * h2);
                const double a2 = 2. * h3 * (g2 * h3 - g3 * h2) / ca, b2 = 2. * h3 * (h2 * f3 - h3 * f2) / ca;
                const double cc2 = 2. * h3 * (f2 * g3 - f3 * g2) / ca;
                c2[ax][0][j] = a2; c2[ax][1][j] = b2; c2[ax][2][j] = cc2;
                c2[ax][3][j] = -(dxp1 * a2 + dxm1 * b2 + dxp2 * cc2) / dxm2;
            }
            {   // first derivative (T:439-504)
                const double f1 = dxp1 + ipow4(dxp1) / ipow3(dxm2), f2 = ipow2(dxp1) - ipow4(dxp1) / ipow2(dxm2),
                             f3 = ipow3(dxp1) + ipow4(dxp1) / dxm2;
                const double g1 = dxm1 - ipow4(dxm1) / ipow3(dxm2), g2 = -ipow2(dxm1) + ipow4(dxm1) / ipow2(dxm2),
                             g3 = ipow3(dxm1) - ipow4(dxm1) / dxm2;
                const double h1 = dxp2 + ipow4(dxp2) / ipow3(dxm2), h2 = ipow2(dxp2) - ipow4(dxp2) / ipow2(dxm2),
                             h3 = ipow3(dxp2) + ipow4(dxp2) / dxm2;
                const double ca = (f1 * h3 - f3 * h1) * (g2 * h3 - g3 * h2) - (g1 * h3 - g3 * h1) * (f2 * h3 - f3 * h2);
                const double a1 = h3 * (g2 * h3 - g3 * h2) / ca, b1 = h3 * (h2 * f3 - h3 * f2) / ca,
                             cc1 = h3 * (f2 * g3 - f3 * g2) / ca;
                c1[ax][0][j] = a1; c1[ax][1][j] = b1; c1[ax][2][j] = cc1;
                c1[ax][3][j] = (ipow2(dxp1) * a1 - ipow2(dxm1) * b1 + ipow2(dxp2) * cc1) / ipow2(dxm2);
            }
        }
    }
    for (int q = 0; q < 3; ++q) cp[q].assign(L[0], 0.);
    for (int j = d.xfirst; j <= d.xlast - 3; ++j) {
        const double dxp1 = xx[j + 1] - xx[j], dxp2 = xx[j + 2] - xx[j], dxp3 = xx[j + 3] - xx[j];
        const double f1 = dxp1 - ipow3(dxp1) / ipow2(dxp3), f2 = ipow2(dxp1) - ipow3(dxp1) / dxp3;
        const double g1 = dxp2 - ipow3(dxp2) / ipow2(dxp3), g2 = ipow2(dxp2) - ipow3(dxp2) / dxp3;
        const double ca = f1 * g2 - f2 * g1;
        cp[0][j] = g2 / ca;
        cp[1][j] = -f2 / ca;
        cp[2][j] = (1 - cp[0][j] * dxp1 - cp[1][j] * dxp2) / dxp3;
    }
    std::vector<std::vector<double>> out{xx, yy, zz, dx, dy, dz};
    for (int ax = 0; ax < 3; ++ax) for (int q = 0; q < 4; ++q) out.push_back(c1[ax][q]);
    for (int ax = 0; ax < 3; ++ax) for (int q = 0; q < 4; ++q) out.push_back(c2[ax][q]);
    for (int q = 0; q < 3; ++q) out.push_back(cp[q]);
    return out;
}

// Tables from NTAB pointers in the order of make_tables
inline void bind_tables(Tables& t, const double* const* p) {
    int o = 0;
    t.xx = p[o++]; t.yy = p[o++]; t.zz = p[o++]; t.dx = p[o++]; t.dy = p[o++]; t.dz = p[o++];
    const double** d1[12] = {&t.ax1, &t.bx1, &t.cx1, &t.dx1, &t.ay1, &t.by1, &t.cy1, &t.dy1, &t.az1, &t.bz1, &t.cz1, &t.dz1};
    const double** d2[12] = {&t.ax2, &t.bx2, &t.cx2, &t.dx2, &t.ay2, &t.by2, &t.cy2, &t.dy2, &t.az2, &t.bz2, &t.cz2, &t.dz2};
    for (auto* q : d1) *q = p[o++];
    for (auto* q : d2) *q = p[o++];
    t.axp = p[o++]; t.bxp = p[o++]; t.cxp = p[o++];
}

// r of every physical node, zero elsewhere (initia, T:771-776; rr0 and rr1 alike, the centre of
// rr1 at x = 0.0); tab: the tables of make_tables
inline std::vector<double> make_radius(const Dims& d, const std::vector<std::vector<double>>& tab) {
    const std::vector<double>&xx = tab[0], &yy = tab[1], &zz = tab[2];
    std::vector<double> r(d.n, 0.);
    for (int jz = 3; jz <= d.mz + 2; ++jz)
        for (int jy = 1; jy <= d.my; ++jy)
            for (int jx = 3; jx <= d.mx + 2; ++jx)
                r[d.at(jx, jy, jz)] = std::sqrt(xx[jx] * xx[jx] + yy[jy] * yy[jy] + zz[jz] * zz[jz]);
    return r;
}

// Fields of one context, carved from consecutive blocks: take(k) returns k fields
template <class Take>
inline void carve(Arr& a, Take take) {
    a.x = take(8); a.xm = take(8); a.xfold = take(8); a.xdif = take(8);
    a.cur = take(3); a.efld = take(3); a.xdh = take(3); a.xresd = take(3);
    a.w = take(1); a.fs = take(1); a.gs = take(1); a.hs = take(1); a.u = take(1); a.v = take(1);
    a.rhoi = take(1); a.bxi = take(1); a.byi = take(1); a.bzi = take(1); a.pri = take(1);
    a.rr0 = take(1); a.rr1 = take(1);
}
constexpr int NFIELDS = 4 * 8 + 4 * 3 + 6 + 7;   // fields carve takes

}  // namespace walls
}  // namespace dasha
