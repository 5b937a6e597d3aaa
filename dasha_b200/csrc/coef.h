// coef.h -- 4th-order 5-point stencil weights on a non-uniform grid (host, FP64).
#pragma once
#include <cmath>
#include <utility>

namespace dasha {
// ---------------------------------------------------------------------------------------
// Stencil coefficients.  The reference builds its 5-point coefficients from closed forms
// (first derivative t3dsdsc.f:439-504, second derivative t3dsdsc.f:336-437).  Both are the
// unique 5-point weights a,b,c,d of
//     D f = a (f+ - f0) + b (f0 - f-) + c (f++ - f0) + d (f0 - f--)
// that are exact for (x - x0)^n, n = 1..4 (n=1 -> 1 for the first derivative, n=2 -> 2 for
// the second).  Here they are obtained by solving that 4x4 system directly (partial
// pivoting), an independent route to the same numbers.
inline bool solve4(double A[4][4], double rhs[4], double out[4]) {
    double M[4][5];
    for (int r = 0; r < 4; ++r) { for (int c = 0; c < 4; ++c) M[r][c] = A[r][c]; M[r][4] = rhs[r]; }
    for (int c = 0; c < 4; ++c) {
        int best = c;
        for (int r = c + 1; r < 4; ++r) if (std::fabs(M[r][c]) > std::fabs(M[best][c])) best = r;
        if (M[best][c] == 0.0) return false;
        if (best != c) for (int q = 0; q < 5; ++q) std::swap(M[best][q], M[c][q]);
        for (int r = c + 1; r < 4; ++r) {
            double f = M[r][c] / M[c][c];
            for (int q = c; q < 5; ++q) M[r][q] -= f * M[c][q];
        }
    }
    for (int r = 3; r >= 0; --r) {
        double s = M[r][4];
        for (int q = r + 1; q < 4; ++q) s -= M[r][q] * out[q];
        out[r] = s / M[r][r];
    }
    return true;
}

// offsets hp1 = x+1 - x0, hm1 = x0 - x-1, hp2 = x+2 - x0, hm2 = x0 - x-2 (all > 0)
inline bool stencil_weights(double hp1, double hm1, double hp2, double hm2, int order, double w[4]) {
    double A[4][4], b[4];
    for (int n = 1; n <= 4; ++n) {
        A[n - 1][0] = std::pow(hp1, n);
        A[n - 1][1] = -std::pow(-hm1, n);
        A[n - 1][2] = std::pow(hp2, n);
        A[n - 1][3] = -std::pow(-hm2, n);
        b[n - 1] = (order == 1) ? (n == 1 ? 1.0 : 0.0) : (n == 2 ? 2.0 : 0.0);
    }
    return solve4(A, b, w);
}


}  // namespace dasha
