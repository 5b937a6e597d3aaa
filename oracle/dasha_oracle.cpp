/*
 * CPU FP64 ORACLE -- TEST INFRASTRUCTURE ONLY.
 *
 * This file restates, in plain C++ (FP64, scalar loops, optional OpenMP), the RK4
 * finite-difference Hall-MHD time step of the reference Fortran program t3dsdsc.f
 * (with its include files mhd01.for, mhd02.for, mhd03.for).  It is the oracle the tests compare
 * the CUDA library in dasha_b200/ with: only tests/, __graft_entry__.smoke() and the cpu_baseline /
 * reference leg of bench.py may load it.  The product never links or calls it.
 *
 * PINNED AGAINST THE REFERENCE ITSELF.  The reference ships no tests, golden vectors or
 * fixtures, and no Fortran compiler exists on these machines; its own source is instead
 * translated to C (oracle/f77c.py) and built under oracle/_ref/ (oracle/refmodel.py), and
 * tests/test_reference_pin.py runs the reference's input, right, current, setdt and stepon
 * beside this restatement on the same nodes and state: stencil coefficients, one right-hand
 * side (Hall on and off, uniform and stretched z), the smoothed current, dt, and one RK4 step
 * with the post-step filter agree to 1e-13..1e-16 of each field's scale on every node that the
 * two codes' different x/y boundary handling cannot reach (the reference's periodic branches
 * are defective, so it runs with its x/y walls there).  Known-answer tests derived from the
 * reference's formulas (polynomial exactness of the stencil coefficients, difc on uniform
 * grids, equilibrium preservation, conservation, symmetry) in tests/ pin the rest.
 *
 * Semantics of the one-domain build (the reference's 1x1 process grid):
 *   node (i,j,k), 0-based, x fastest, is the reference's (jx,jy,jz) = (i+3, j+1, k+3);
 *   x and y are periodic with a true wrap (every node interior);  z has walls: rows
 *   k = 2 .. mz-3 are interior (the reference's z_first..z_last = 5..mz, T:74-79) and the
 *   rows k = 0,1 and mz-2,mz-1 follow the reference's fixed rows (outer row 0, next row
 *   one half of its inner neighbour; e.g. bndry T:1821-1857).
 * The reference's periodic branches (T:1787-1818 and the like) copy one stale ghost row
 * only; a correct wrap is used instead.  Dipole-only code (inflow driver T:1710-1773,
 * inner-sphere mask T:1692-1707, radial Hall profile T:1398, the totalE=.false. branch
 * T:1464-1547) is not part of this restatement.
 */
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" {

/* Same field order and meaning as the library's dasha_params_c. */
typedef struct {
    double gamma, eta, di, mu, drho, dp, cfl, rcr;
    int hall, viscos, diffu, total_e, j0_mode;
    int filter_every;
    int precision;
    int dt_whistler;
} oracle_params;

}

namespace {

typedef std::vector<double> vec;

/* d1fc / d2fc statement functions, T:1308-1313: a*(f+ - f0) + b*(f0 - f-) + c*(f++ - f0)
 * + d*(f0 - f--), evaluated left to right as Fortran does. */
inline double d1fc(double fm2, double fm, double f0, double fp, double fp2,
                   double a, double b, double c, double d) {
    return a * (fp - f0) + b * (f0 - fm) + c * (fp2 - f0) + d * (f0 - fm2);
}

/* difc statement function of the smoothing routines, T:5618-5619. */
inline double difc(double fm, double f0, double fp, double xm1, double x0, double xp1) {
    return 2. * ((fp - f0) * (xp1 - x0) - (f0 - fm) * (x0 - xm1)) / (xp1 - xm1);
}

struct Oracle {
    int mx, my, mz;
    long N, sy, sz;
    vec xc, yc, zc;          /* node coordinates */
    double Lx, Ly;           /* periods of x and y */
    oracle_params P;
    /* neighbour tables (periodic wrap) */
    std::vector<int> xi[5], yj[5];   /* index of i-2..i+2 */
    vec xext[5], yext[5];            /* coordinate of i-2..i+2 continued across the wrap */
    /* 1st- and 2nd-derivative coefficients, T:336-504; zero where undefined */
    vec ax1, bx1, cx1, dx1, ay1, by1, cy1, dy1, az1, bz1, cz1, dz1;
    vec ax2, bx2, cx2, dx2, ay2, by2, cy2, dy2, az2, bz2, cz2, dz2;
    /* equilibrium (3-D like rhoi/bxi/byi/bzi/pri, T:805-813) and J0 for j0_mode FULL */
    vec rhoi, bxi, byi, bzi, pri, j0[3];
    vec xresd[3];
    vec x[8], xm[8], xfold[8], xdif[8], cur[3], efld[3], xdh[3];
    vec fs, gs, hs, w, u3, v3, w3;
    vec cr;                  /* radial smoothing coefficient per node (T:5659-5661) */
    vec cbx;                 /* x-only coefficient for B in avrg/avrgtt (T:5636-5642) */

    inline long id(int i, int j, int k) const { return i + sy * j + sz * k; }

    /* ---- derivatives (interior nodes) ---- */
    inline double Dx(const vec& f, int i, int j, int k) const {
        long b = sy * j + sz * k;
        return d1fc(f[b + xi[0][i]], f[b + xi[1][i]], f[b + i], f[b + xi[3][i]], f[b + xi[4][i]],
                    ax1[i], bx1[i], cx1[i], dx1[i]);
    }
    inline double Dy(const vec& f, int i, int j, int k) const {
        long b = i + sz * k;
        return d1fc(f[b + sy * yj[0][j]], f[b + sy * yj[1][j]], f[b + sy * j], f[b + sy * yj[3][j]],
                    f[b + sy * yj[4][j]], ay1[j], by1[j], cy1[j], dy1[j]);
    }
    inline double Dz(const vec& f, int i, int j, int k) const {
        long c = id(i, j, k);
        return d1fc(f[c - 2 * sz], f[c - sz], f[c], f[c + sz], f[c + 2 * sz],
                    az1[k], bz1[k], cz1[k], dz1[k]);
    }
    inline double D2x(const vec& f, int i, int j, int k) const {
        long b = sy * j + sz * k;
        return d1fc(f[b + xi[0][i]], f[b + xi[1][i]], f[b + i], f[b + xi[3][i]], f[b + xi[4][i]],
                    ax2[i], bx2[i], cx2[i], dx2[i]);
    }
    inline double D2y(const vec& f, int i, int j, int k) const {
        long b = i + sz * k;
        return d1fc(f[b + sy * yj[0][j]], f[b + sy * yj[1][j]], f[b + sy * j], f[b + sy * yj[3][j]],
                    f[b + sy * yj[4][j]], ay2[j], by2[j], cy2[j], dy2[j]);
    }
    inline double D2z(const vec& f, int i, int j, int k) const {
        long c = id(i, j, k);
        return d1fc(f[c - 2 * sz], f[c - sz], f[c], f[c + sz], f[c + 2 * sz],
                    az2[k], bz2[k], cz2[k], dz2[k]);
    }
    /* sum of the three difc terms of one smoothing pass, T:5643-5648 */
    inline double difc3(const vec& f, int i, int j, int k) const {
        long c = id(i, j, k);
        long b = sy * j + sz * k;
        double tx = difc(f[b + xi[1][i]], f[c], f[b + xi[3][i]], xext[1][i], xc[i], xext[3][i]);
        long by_ = i + sz * k;
        double ty = difc(f[by_ + sy * yj[1][j]], f[c], f[by_ + sy * yj[3][j]], yext[1][j], yc[j], yext[3][j]);
        double tz = difc(f[c - sz], f[c], f[c + sz], zc[k - 1], zc[k], zc[k + 1]);
        return tx + ty + tz;
    }

    /* ---- grid and coefficients ---- */
    void init_grid() {
        Lx = xc[mx - 1] - xc[0] + (xc[1] - xc[0]);   /* periodic continuation, cf. T:278-283 */
        Ly = yc[my - 1] - yc[0] + (yc[1] - yc[0]);
        for (int o = 0; o < 5; ++o) {
            xi[o].resize(mx); xext[o].resize(mx);
            yj[o].resize(my); yext[o].resize(my);
            for (int i = 0; i < mx; ++i) {
                int ii = i + o - 2, q = 0;
                while (ii < 0) { ii += mx; --q; }
                while (ii >= mx) { ii -= mx; ++q; }
                xi[o][i] = ii; xext[o][i] = xc[ii] + q * Lx;
            }
            for (int j = 0; j < my; ++j) {
                int jj = j + o - 2, q = 0;
                while (jj < 0) { jj += my; --q; }
                while (jj >= my) { jj -= my; ++q; }
                yj[o][j] = jj; yext[o][j] = yc[jj] + q * Ly;
            }
        }
        auto alloc = [](vec& v, int n) { v.assign(n, 0.0); };
        for (vec* v : {&ax1, &bx1, &cx1, &dx1, &ax2, &bx2, &cx2, &dx2}) alloc(*v, mx);
        for (vec* v : {&ay1, &by1, &cy1, &dy1, &ay2, &by2, &cy2, &dy2}) alloc(*v, my);
        for (vec* v : {&az1, &bz1, &cz1, &dz1, &az2, &bz2, &cz2, &dz2}) alloc(*v, mz);
        for (int i = 0; i < mx; ++i)
            coef_node(xext[3][i] - xc[i], xc[i] - xext[1][i], xext[4][i] - xc[i], xc[i] - xext[0][i],
                      ax1[i], bx1[i], cx1[i], dx1[i], ax2[i], bx2[i], cx2[i], dx2[i]);
        for (int j = 0; j < my; ++j)
            coef_node(yext[3][j] - yc[j], yc[j] - yext[1][j], yext[4][j] - yc[j], yc[j] - yext[0][j],
                      ay1[j], by1[j], cy1[j], dy1[j], ay2[j], by2[j], cy2[j], dy2[j]);
        for (int k = 2; k <= mz - 3; ++k)   /* z_first..z_last only, T:406 / T:483 */
            coef_node(zc[k + 1] - zc[k], zc[k] - zc[k - 1], zc[k + 2] - zc[k], zc[k] - zc[k - 2],
                      az1[k], bz1[k], cz1[k], dz1[k], az2[k], bz2[k], cz2[k], dz2[k]);
        cr.assign(N, 0.0);
        cbx.assign(mx, 0.0);
        for (int k = 0; k < mz; ++k)
            for (int j = 0; j < my; ++j)
                for (int i = 0; i < mx; ++i) {
                    double r = std::sqrt(xc[i] * xc[i] + yc[j] * yc[j] + zc[k] * zc[k]);
                    /* T:5659-5661 (coef_avrg of avrg / avrgtt / avrgE / avrgc) */
                    cr[id(i, j, k)] = 1.0 / 32.0 + (1.0 / 8.0 - 1.0 / 32.0) * 0.5 * (1 + std::tanh((r - 3.) / 3.));
                }
        for (int i = 0; i < mx; ++i) cbx[i] = 1 - std::tanh((xc[i] + 3) / 8.);   /* T:5642 */
    }

    /* One node's coefficients: second derivative T:337-364, first derivative T:440-459. */
    static void coef_node(double dxp1, double dxm1, double dxp2, double dxm2,
                          double& a1, double& b1, double& c1, double& d1,
                          double& a2, double& b2, double& c2, double& d2) {
        {
            double f1 = dxp1 * dxp1 + dxp1 * dxm2;
            double f2 = dxp1 * dxp1 * dxp1 - dxp1 * dxm2 * dxm2;
            double f3 = std::pow(dxp1, 4) + dxp1 * std::pow(dxm2, 3);
            double g1 = -dxm1 * dxm1 + dxm1 * dxm2;
            double g2 = std::pow(dxm1, 3) - dxm1 * dxm2 * dxm2;
            double g3 = -std::pow(dxm1, 4) + dxm1 * std::pow(dxm2, 3);
            double h1 = dxp2 * dxp2 + dxp2 * dxm2;
            double h2 = std::pow(dxp2, 3) - dxp2 * dxm2 * dxm2;
            double h3 = std::pow(dxp2, 4) + dxp2 * std::pow(dxm2, 3);
            double ca = (f1 * h3 - f3 * h1) * (g2 * h3 - g3 * h2) - (g1 * h3 - g3 * h1) * (f2 * h3 - f3 * h2);
            (void)g1;
            a2 = 2. * h3 * (g2 * h3 - g3 * h2) / ca;
            b2 = 2. * h3 * (h2 * f3 - h3 * f2) / ca;
            c2 = 2. * h3 * (f2 * g3 - f3 * g2) / ca;
            d2 = -(dxp1 * a2 + dxm1 * b2 + dxp2 * c2) / dxm2;
        }
        {
            double f1 = dxp1 + std::pow(dxp1, 4) / std::pow(dxm2, 3);
            double f2 = dxp1 * dxp1 - std::pow(dxp1, 4) / (dxm2 * dxm2);
            double f3 = std::pow(dxp1, 3) + std::pow(dxp1, 4) / dxm2;
            double g1 = dxm1 - std::pow(dxm1, 4) / std::pow(dxm2, 3);
            double g2 = -dxm1 * dxm1 + std::pow(dxm1, 4) / (dxm2 * dxm2);
            double g3 = std::pow(dxm1, 3) - std::pow(dxm1, 4) / dxm2;
            double h1 = dxp2 + std::pow(dxp2, 4) / std::pow(dxm2, 3);
            double h2 = dxp2 * dxp2 - std::pow(dxp2, 4) / (dxm2 * dxm2);
            double h3 = std::pow(dxp2, 3) + std::pow(dxp2, 4) / dxm2;
            double ca = (f1 * h3 - f3 * h1) * (g2 * h3 - g3 * h2) - (g1 * h3 - g3 * h1) * (f2 * h3 - f3 * h2);
            a1 = h3 * (g2 * h3 - g3 * h2) / ca;
            b1 = h3 * (h2 * f3 - h3 * f2) / ca;
            c1 = h3 * (f2 * g3 - f3 * g2) / ca;
            d1 = (dxp1 * dxp1 * a1 - dxm1 * dxm1 * b1 + dxp2 * dxp2 * c1) / (dxm2 * dxm2);
        }
    }

    /* ---- fixed z rows (bndry T:1821-1857, bndrytt T:2131-2167, bndryc T:2614-2642,
     *      bndryh T:2782-2815, bndryE T:2946-2975) ---- */
    void zrows(vec& f) {
        for (int j = 0; j < my; ++j)
            for (int i = 0; i < mx; ++i) {
                f[id(i, j, 0)] = 0.;
                f[id(i, j, 1)] = 0.5 * f[id(i, j, 2)];
                f[id(i, j, mz - 1)] = 0.;
                f[id(i, j, mz - 2)] = 0.5 * f[id(i, j, mz - 3)];
            }
    }

    /* One Jacobi smoothing pass on the interior of f: f += coef * (difc_x + difc_y + difc_z).
     * kind 0: radial coef (avrgc T:5981-5992, avrgE T:5895-5906, avrg/avrgtt non-B T:5659-5670);
     * kind 1: 1/8 (avrgh T:6031-6042);  kind 2: x-profile for B (avrg/avrgtt T:5636-5648). */
    void smooth_pass(vec& f, int kind) {
#pragma omp parallel for schedule(static)
        for (int k = 2; k <= mz - 3; ++k)
            for (int j = 0; j < my; ++j)
                for (int i = 0; i < mx; ++i) {
                    long c = id(i, j, k);
                    double s = difc3(f, i, j, k);
                    double val;
                    if (kind == 0) val = f[c] + cr[c] * s;
                    else if (kind == 1) val = f[c] + (1.0 / 8.0) * s;
                    else val = f[c] + (1 - 0.0) * (1.0 / 32.0) * cbx[i] * s;
                    w[c] = val;
                }
        for (int k = 2; k <= mz - 3; ++k)
            std::memcpy(&f[id(0, 0, k)], &w[id(0, 0, k)], sizeof(double) * sz);
    }

    /* ---- current, T:2452-2500 ---- */
    void current() {
#pragma omp parallel for schedule(static)
        for (long c = 0; c < N; ++c) {
            u3[c] = x[4][c] - bxi[c];
            v3[c] = x[5][c] - byi[c];
            w3[c] = x[6][c] - bzi[c];
        }
#pragma omp parallel for schedule(static)
        for (int k = 2; k <= mz - 3; ++k)
            for (int j = 0; j < my; ++j)
                for (int i = 0; i < mx; ++i) {
                    long c = id(i, j, k);
                    cur[0][c] = Dy(w3, i, j, k) - Dz(v3, i, j, k);
                    cur[1][c] = Dz(u3, i, j, k) - Dx(w3, i, j, k);
                    cur[2][c] = Dx(v3, i, j, k) - Dy(u3, i, j, k);
                }
        for (int m = 0; m < 3; ++m) zrows(cur[m]);          /* bndryc */
        for (int pass = 0; pass < 4; ++pass) {               /* avrgc(1,3,4) T:2495 */
            for (int m = 0; m < 3; ++m) smooth_pass(cur[m], 0);
            for (int m = 0; m < 3; ++m) zrows(cur[m]);
        }
        if (P.j0_mode == 1)
            for (int m = 0; m < 3; ++m)
                for (long c = 0; c < N; ++c) cur[m][c] += j0[m][c];
    }

    /* ---- flux(m), m=1..4, T:2304-2347 (0-based m here) ---- */
    void flux(int m) {
#pragma omp parallel for schedule(static)
        for (long c = 0; c < N; ++c) {
            const double r = x[0][c];
            if (m == 0) {
                fs[c] = x[1][c]; gs[c] = x[2][c]; hs[c] = x[3][c];
            } else if (m == 1) {
                fs[c] = x[1][c] * x[1][c] / r + (x[7][c] - pri[c]);
                gs[c] = x[1][c] * x[2][c] / r;
                hs[c] = x[1][c] * x[3][c] / r;
            } else if (m == 2) {
                fs[c] = x[1][c] * x[2][c] / r;
                gs[c] = x[2][c] * x[2][c] / r + (x[7][c] - pri[c]);
                hs[c] = x[3][c] * x[2][c] / r;
            } else {
                fs[c] = x[1][c] * x[3][c] / r;
                gs[c] = x[2][c] * x[3][c] / r;
                hs[c] = x[3][c] * x[3][c] / r + (x[7][c] - pri[c]);
            }
        }
    }

    /* ---- right(t), T:1297-1673 ---- */
    void right(double t) {
        const double eta = P.eta, gamma = P.gamma;
        current();
        for (int m = 0; m < 4; ++m) {
            flux(m);
#pragma omp parallel for schedule(static)
            for (int k = 2; k <= mz - 3; ++k)
                for (int j = 0; j < my; ++j)
                    for (int i = 0; i < mx; ++i)
                        xdif[m][id(i, j, k)] = -Dx(fs, i, j, k) - Dy(gs, i, j, k) - Dz(hs, i, j, k);
        }
        /* all points, T:1348-1387 (totalE = .true.) */
#pragma omp parallel for schedule(static)
        for (long c = 0; c < N; ++c) {
            const double r = x[0][c];
            fs[c] = x[1][c] / r; gs[c] = x[2][c] / r; hs[c] = x[3][c] / r;
            xdif[1][c] = xdif[1][c] - xresd[0][c] + cur[1][c] * x[6][c] - cur[2][c] * x[5][c];
            xdif[2][c] = xdif[2][c] - xresd[1][c] + cur[2][c] * x[4][c] - cur[0][c] * x[6][c];
            xdif[3][c] = xdif[3][c] - xresd[2][c] + cur[0][c] * x[5][c] - cur[1][c] * x[4][c];
            efld[0][c] = (-x[2][c] * x[6][c] + x[3][c] * x[5][c]) / r + eta * cur[0][c];
            efld[1][c] = (-x[3][c] * x[4][c] + x[1][c] * x[6][c]) / r + eta * cur[1][c];
            efld[2][c] = (-x[1][c] * x[5][c] + x[2][c] * x[4][c]) / r + eta * cur[2][c];
        }
        for (int pass = 0; pass < 4; ++pass) {               /* avrgE(t,1,3,4) T:1389 */
            for (int m = 0; m < 3; ++m) smooth_pass(efld[m], 0);
            for (int m = 0; m < 3; ++m) zrows(efld[m]);
        }
        if (P.hall) {                                         /* T:1391-1433, cht = di */
            const double cht = P.di;
#pragma omp parallel for schedule(static)
            for (int k = 2; k <= mz - 3; ++k)
                for (int j = 0; j < my; ++j)
                    for (int i = 0; i < mx; ++i) {
                        long c = id(i, j, k);
                        const vec& p = x[7];
                        xdh[0][c] = cht * (cur[1][c] * x[6][c] - cur[2][c] * x[5][c] - Dx(p, i, j, k)) / x[0][c];
                        xdh[1][c] = cht * (cur[2][c] * x[4][c] - cur[0][c] * x[6][c] - Dy(p, i, j, k)) / x[0][c];
                        xdh[2][c] = cht * (cur[0][c] * x[5][c] - cur[1][c] * x[4][c] - Dz(p, i, j, k)) / x[0][c];
                    }
            for (int m = 0; m < 3; ++m) zrows(xdh[m]);       /* bndryh */
            for (int pass = 0; pass < 5; ++pass) {           /* avrgh(1,3,5) */
                for (int m = 0; m < 3; ++m) smooth_pass(xdh[m], 1);
                for (int m = 0; m < 3; ++m) zrows(xdh[m]);
            }
            for (int m = 0; m < 3; ++m)
                for (long c = 0; c < N; ++c) efld[m][c] = efld[m][c] + xdh[m][c];
        }
        /* induction and pressure, T:1435-1566 */
#pragma omp parallel for schedule(static)
        for (int k = 2; k <= mz - 3; ++k)
            for (int j = 0; j < my; ++j)
                for (int i = 0; i < mx; ++i) {
                    long c = id(i, j, k);
                    xdif[4][c] = -Dy(efld[2], i, j, k) + Dz(efld[1], i, j, k);
                    xdif[5][c] = -Dz(efld[0], i, j, k) + Dx(efld[2], i, j, k);
                    xdif[6][c] = -Dx(efld[1], i, j, k) + Dy(efld[0], i, j, k);
                    const vec& p = x[7];
                    double c2 = cur[0][c] * cur[0][c] + cur[1][c] * cur[1][c] + cur[2][c] * cur[2][c];
                    xdif[7][c] = -Dx(p, i, j, k) * fs[c] - Dy(p, i, j, k) * gs[c] - Dz(p, i, j, k) * hs[c]
                               + (-Dx(fs, i, j, k) - Dy(gs, i, j, k) - Dz(hs, i, j, k)) * gamma * p[c]
                               + (gamma - 1.) * eta * c2;
                }
        if (P.viscos) {                                       /* T:1585-1636 */
#pragma omp parallel for schedule(static)
            for (int k = 2; k <= mz - 3; ++k)
                for (int j = 0; j < my; ++j)
                    for (int i = 0; i < mx; ++i) {
                        long c = id(i, j, k);
                        double af = D2x(fs, i, j, k) + D2y(fs, i, j, k) + D2z(fs, i, j, k);
                        double ag = D2x(gs, i, j, k) + D2y(gs, i, j, k) + D2z(gs, i, j, k);
                        double ah = D2x(hs, i, j, k) + D2y(hs, i, j, k) + D2z(hs, i, j, k);
                        xdif[1][c] = xdif[1][c] + P.mu * af;
                        xdif[2][c] = xdif[2][c] + P.mu * ag;
                        xdif[3][c] = xdif[3][c] + P.mu * ah;
                        xdif[7][c] = xdif[7][c] + P.mu * (fs[c] * af + gs[c] * ag + hs[c] * ah);
                    }
        }
        if (P.diffu) {                                        /* T:1638-1663 */
#pragma omp parallel for schedule(static)
            for (int k = 2; k <= mz - 3; ++k)
                for (int j = 0; j < my; ++j)
                    for (int i = 0; i < mx; ++i) {
                        long c = id(i, j, k);
                        xdif[0][c] = xdif[0][c] + P.drho * (D2x(x[0], i, j, k) + D2y(x[0], i, j, k) + D2z(x[0], i, j, k));
                        xdif[7][c] = xdif[7][c] + P.dp * (D2x(x[7], i, j, k) + D2y(x[7], i, j, k) + D2z(x[7], i, j, k));
                    }
        }
        for (int m = 0; m < 8; ++m) zrows(xdif[m]);          /* bndry T:1665 */
        if (t != 0.) {                                        /* avrg(t,ddt,km,1,8,0,2) T:1669 */
            for (int pass = 0; pass < 2; ++pass) {
                for (int m = 0; m < 8; ++m) smooth_pass(xdif[m], (m >= 4 && m <= 6) ? 2 : 0);
                for (int m = 0; m < 8; ++m) zrows(xdif[m]);
            }
        }
    }

    /* ---- stepon, T:1063-1172 ---- */
    void stepon(double time, double dt, int nstep) {
        for (int m = 0; m < 8; ++m) xfold[m] = x[m];
        right(time + dt / 2);
        for (int m = 0; m < 8; ++m)
#pragma omp parallel for schedule(static)
            for (long c = 0; c < N; ++c) {
                xm[m][c] = xfold[m][c] + xdif[m][c] * dt / 6.;
                x[m][c] = xfold[m][c] + xdif[m][c] * dt / 2.;
            }
        right(time + dt / 2);
        for (int m = 0; m < 8; ++m)
#pragma omp parallel for schedule(static)
            for (long c = 0; c < N; ++c) {
                xm[m][c] = xm[m][c] + xdif[m][c] * dt / 3.;
                x[m][c] = xfold[m][c] + xdif[m][c] * dt / 2.;
            }
        right(time + dt);
        for (int m = 0; m < 8; ++m)
#pragma omp parallel for schedule(static)
            for (long c = 0; c < N; ++c) {
                xm[m][c] = xm[m][c] + xdif[m][c] * dt / 3.;
                x[m][c] = xfold[m][c] + xdif[m][c] * dt;
            }
        right(time + dt);
        for (int m = 0; m < 8; ++m)
#pragma omp parallel for schedule(static)
            for (long c = 0; c < N; ++c) x[m][c] = xm[m][c] + xdif[m][c] * dt / 6.;
        int every = P.filter_every > 0 ? P.filter_every : 1;
        if (nstep % every == 0) {
            /* T:1135-1165: filter the perturbation x - eq with avrgtt(tt,1,8,0,2) */
            for (long c = 0; c < N; ++c) {
                xm[0][c] = x[0][c] - rhoi[c];
                xm[1][c] = x[1][c]; xm[2][c] = x[2][c]; xm[3][c] = x[3][c];
                xm[4][c] = x[4][c] - bxi[c];
                xm[5][c] = x[5][c] - byi[c];
                xm[6][c] = x[6][c] - bzi[c];
                xm[7][c] = x[7][c] - pri[c];
            }
            for (int pass = 0; pass < 2; ++pass) {           /* avrgtt T:5770-5821 */
                for (int m = 0; m < 8; ++m) smooth_pass(xm[m], (m >= 4 && m <= 6) ? 2 : 0);
                for (int m = 0; m < 8; ++m) zrows(xm[m]);    /* bndrytt */
            }
            for (long c = 0; c < N; ++c) {
                x[0][c] = xm[0][c] + rhoi[c];
                x[1][c] = xm[1][c]; x[2][c] = xm[2][c]; x[3][c] = xm[3][c];
                x[4][c] = xm[4][c] + bxi[c];
                x[5][c] = xm[5][c] + byi[c];
                x[6][c] = xm[6][c] + bzi[c];
                x[7][c] = xm[7][c] + pri[c];
            }
        }
    }

    /* ---- setdt, T:4694-4763 (the asymmetric region of T:4709-4711 is kept) ---- */
    double setdt() const {
        double dtt = 100.;
        const double eta = P.eta, fmu = P.mu, cfl = P.cfl, gamma = P.gamma;
        for (int k = 0; k <= mz - 3; ++k)
            for (int j = 0; j <= my - 2; ++j)
                for (int i = 0; i <= mx - 3; ++i) {
                    long c = id(i, j, k);
                    double r = std::sqrt(xc[i] * xc[i] + yc[j] * yc[j] + zc[k] * zc[k]);
                    if (!(r >= P.rcr)) continue;
                    double vx = x[1][c] / x[0][c], vy = x[2][c] / x[0][c], vz = x[3][c] / x[0][c];
                    double va2 = (x[4][c] * x[4][c] + x[5][c] * x[5][c] + x[6][c] * x[6][c]) / x[0][c];
                    double cs2 = gamma * x[7][c] / x[0][c];
                    double vpx = std::fabs(vx) + std::sqrt(std::fabs(va2 + cs2));
                    double vpy = std::fabs(vy) + std::sqrt(std::fabs(va2 + cs2));
                    double vpz = std::fabs(vz) + std::sqrt(std::fabs(va2 + cs2));
                    double dxi = xext[3][i] - xc[i], dyj = yext[3][j] - yc[j], dzk = zc[k + 1] - zc[k];
                    if (P.dt_whistler && P.hall) {   /* build option: grid-scale whistler speed */
                        double bm = std::sqrt(x[4][c] * x[4][c] + x[5][c] * x[5][c] + x[6][c] * x[6][c]);
                        double w = P.di * 3.141592653589793 * bm / x[0][c];
                        vpx += w / std::fabs(dxi); vpy += w / std::fabs(dyj); vpz += w / std::fabs(dzk);
                    }
                    double dtx = std::fabs(dxi) / (vpx / cfl + (eta + fmu) / dxi / 2.);
                    double dty = std::fabs(dyj) / (vpy / cfl + (eta + fmu) / dyj / 2.);
                    double dtz = std::fabs(dzk) / (vpz / cfl + (eta + fmu) / dzk / 2.);
                    double dt1 = std::min(dtx, dty);
                    double dt2 = std::min(dtz, dt1);
                    dtt = std::min(dtt, dt2);
                }
        return dtt;
    }

    /* ---- diagnostics: J extrema on the mid-y plane (diagn T:1199-1214, funmax T:6114-6139)
     *      plus FP64 mass, energy and reconnected flux ---- */
    void diagnostics(double* out) {
        current();
        const int jm = my / 2;   /* jy = my/2+1, 1-based */
        double mx_[3], mn_[3];
        for (int m = 0; m < 3; ++m) { mx_[m] = -1000000.; mn_[m] = 1000000.; }
        for (int k = 0; k < mz; ++k)
            for (int i = 0; i < mx; ++i)
                for (int m = 0; m < 3; ++m) {
                    double v = cur[m][id(i, jm, k)];
                    if (v > mx_[m]) mx_[m] = v;
                    if (v < mn_[m]) mn_[m] = v;
                }
        double mass = 0., energy = 0.;
        for (int k = 0; k < mz; ++k) {
            double wz = 0.5 * (zc[std::min(k + 1, mz - 1)] - zc[std::max(k - 1, 0)]);
            double sm = 0., se = 0.;
            for (int j = 0; j < my; ++j) {
                double wy = 0.5 * (yext[3][j] - yext[1][j]);
                for (int i = 0; i < mx; ++i) {
                    double wx = 0.5 * (xext[3][i] - xext[1][i]);
                    long c = id(i, j, k);
                    double vol = wx * wy;
                    double r = x[0][c];
                    double ke = 0.5 * (x[1][c] * x[1][c] + x[2][c] * x[2][c] + x[3][c] * x[3][c]) / r;
                    double me = 0.5 * (x[4][c] * x[4][c] + x[5][c] * x[5][c] + x[6][c] * x[6][c]);
                    sm += r * vol;
                    se += (ke + x[7][c] / (P.gamma - 1.) + me) * vol;
                }
            }
            mass += sm * wz;
            energy += se * wz;
        }
        double flux = 0.;
        const double eps2 = 1e-20;
        for (int j = 0; j < my; ++j)
            for (int i = 0; i < mx; ++i) {
                double bz;
                if (mz % 2) bz = x[6][id(i, j, (mz - 1) / 2)];
                else bz = 0.5 * (x[6][id(i, j, mz / 2 - 1)] + x[6][id(i, j, mz / 2)]);
                double wx = 0.5 * (xext[3][i] - xext[1][i]);
                flux += std::sqrt(bz * bz + eps2) * wx;
            }
        flux /= my;
        out[0] = mass; out[1] = energy; out[2] = flux;
        out[3] = mx_[0]; out[4] = mn_[0]; out[5] = mx_[1]; out[6] = mn_[1]; out[7] = mx_[2]; out[8] = mn_[2];
    }

    /* xresd = momentum RHS of the pure equilibrium state, as initia does it (T:816-834). */
    void init_residual() {
        vec save[8];
        for (int m = 0; m < 8; ++m) save[m] = x[m];
        for (int m = 0; m < 3; ++m) std::fill(xresd[m].begin(), xresd[m].end(), 0.0);
        std::fill(x[1].begin(), x[1].end(), 0.0);
        std::fill(x[2].begin(), x[2].end(), 0.0);
        std::fill(x[3].begin(), x[3].end(), 0.0);
        x[0] = rhoi; x[4] = bxi; x[5] = byi; x[6] = bzi; x[7] = pri;
        for (int m = 0; m < 8; ++m) xfold[m] = x[m];
        right(0.0);
        for (int m = 0; m < 3; ++m) xresd[m] = xdif[m + 1];
        for (int m = 0; m < 8; ++m) x[m] = save[m];
    }
};

}  // namespace

extern "C" {

void* oracle_create(int mx, int my, int mz, const double* x, const double* y, const double* z,
                    const oracle_params* p) {
    if (mx < 5 || my < 5 || mz < 7) return nullptr;
    Oracle* o = new Oracle();
    o->mx = mx; o->my = my; o->mz = mz;
    o->sy = mx; o->sz = (long)mx * my; o->N = o->sz * mz;
    o->xc.assign(x, x + mx); o->yc.assign(y, y + my); o->zc.assign(z, z + mz);
    o->P = *p;
    o->init_grid();
    auto al = [o](vec& v) { v.assign(o->N, 0.0); };
    for (vec* v : {&o->rhoi, &o->bxi, &o->byi, &o->bzi, &o->pri, &o->fs, &o->gs, &o->hs, &o->w,
                   &o->u3, &o->v3, &o->w3}) al(*v);
    for (int m = 0; m < 3; ++m) { al(o->j0[m]); al(o->xresd[m]); al(o->cur[m]); al(o->efld[m]); al(o->xdh[m]); }
    for (int m = 0; m < 8; ++m) { al(o->x[m]); al(o->xm[m]); al(o->xfold[m]); al(o->xdif[m]); }
    return o;
}

void oracle_destroy(void* h) { delete static_cast<Oracle*>(h); }

void oracle_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* Equilibrium as 1-D z profiles: rho0[mz], b0[3*mz] (bx0, by0, bz0), p0[mz], j0[3*mz] or NULL. */
void oracle_set_equilibrium(void* h, const double* rho0, const double* b0, const double* p0, const double* j0) {
    Oracle* o = static_cast<Oracle*>(h);
    for (int k = 0; k < o->mz; ++k)
        for (long c = 0; c < o->sz; ++c) {
            long q = c + o->sz * k;
            o->rhoi[q] = rho0[k];
            o->bxi[q] = b0[k]; o->byi[q] = b0[o->mz + k]; o->bzi[q] = b0[2 * o->mz + k];
            o->pri[q] = p0[k];
            for (int m = 0; m < 3; ++m) o->j0[m][q] = j0 ? j0[m * o->mz + k] : 0.0;
        }
    o->init_residual();
}

/* State as x(mx,my,mz,8) in Fortran order (compact, no halo), total fields. */
void oracle_set_state(void* h, const double* xs) {
    Oracle* o = static_cast<Oracle*>(h);
    for (int m = 0; m < 8; ++m) std::memcpy(o->x[m].data(), xs + m * o->N, sizeof(double) * o->N);
}
void oracle_get_state(void* h, double* xs) {
    Oracle* o = static_cast<Oracle*>(h);
    for (int m = 0; m < 8; ++m) std::memcpy(xs + m * o->N, o->x[m].data(), sizeof(double) * o->N);
}
/* One RHS evaluation right(t) of the current state; xdif(mx,my,mz,8) out. */
void oracle_rhs(void* h, double t, double* out) {
    Oracle* o = static_cast<Oracle*>(h);
    for (int m = 0; m < 8; ++m) { o->xfold[m] = o->x[m]; std::fill(o->xdif[m].begin(), o->xdif[m].end(), 0.0); }
    o->right(t);
    for (int m = 0; m < 8; ++m) std::memcpy(out + m * o->N, o->xdif[m].data(), sizeof(double) * o->N);
}
void oracle_current(void* h, double* out) {
    Oracle* o = static_cast<Oracle*>(h);
    o->current();
    for (int m = 0; m < 3; ++m) std::memcpy(out + m * o->N, o->cur[m].data(), sizeof(double) * o->N);
}
void oracle_residual(void* h, double* out) {
    Oracle* o = static_cast<Oracle*>(h);
    for (int m = 0; m < 3; ++m) std::memcpy(out + m * o->N, o->xresd[m].data(), sizeof(double) * o->N);
}
void oracle_stepon(void* h, double time, double dt, int nstep) {
    static_cast<Oracle*>(h)->stepon(time, dt, nstep);
}
double oracle_setdt(void* h) { return static_cast<Oracle*>(h)->setdt(); }
void oracle_diagnostics(void* h, double* out) { static_cast<Oracle*>(h)->diagnostics(out); }
/* Coefficients for known-answer tests: which = 0 (x), 1 (y), 2 (z); out[8*n]: a1 b1 c1 d1 a2 b2 c2 d2. */
void oracle_coefficients(void* h, int which, double* out) {
    Oracle* o = static_cast<Oracle*>(h);
    int n = which == 0 ? o->mx : which == 1 ? o->my : o->mz;
    const vec* src[3][8] = {
        {&o->ax1, &o->bx1, &o->cx1, &o->dx1, &o->ax2, &o->bx2, &o->cx2, &o->dx2},
        {&o->ay1, &o->by1, &o->cy1, &o->dy1, &o->ay2, &o->by2, &o->cy2, &o->dy2},
        {&o->az1, &o->bz1, &o->cz1, &o->dz1, &o->az2, &o->bz2, &o->cz2, &o->dz2}};
    for (int q = 0; q < 8; ++q) std::memcpy(out + q * n, src[which][q]->data(), sizeof(double) * n);
}
/* One smoothing pass on a caller field (known-answer tests of difc). */
void oracle_smooth_pass(void* h, double* f, int kind) {
    Oracle* o = static_cast<Oracle*>(h);
    vec v(f, f + o->N);
    o->smooth_pass(v, kind);
    std::memcpy(f, v.data(), sizeof(double) * o->N);
}

}  // extern "C"
