// adjoint.cuh -- discrete adjoint (vector-Jacobian products) of the RK4 Hall-MHD step, FP64.
//
// The forward step (stepon, t3dsdsc.f:1063-1185) is X -> F(X + dt/6 (k1 + 2 k2 + 2 k3 + k4))
// with k = G(S) = avrg(right(S)) and F the post-step filter (avrgtt).  With dt held fixed
// (the recorded sequence is replayed) every piece is either linear -- the smoothing passes
// with their wall rows, the curls, the 4th-order derivatives -- or pointwise: E = -v x B +
// eta J, the Hall term, the fluxes and the pressure equation.  Each linear piece is
// transposed here as a gather (one thread per node reads the adjoint at the nodes whose
// stencils touch it); the wall rows y(1) = y(2)/2, y(0) = 0 transpose to a fold of the row
// adjoints into row 2 (and mz-3).  No reference counterpart: the reference has no adjoint.
#pragma once
#include "mhd_kernels.cuh"
#include "zm_kernels.cuh"

namespace dasha {

struct AdjGrid {
    int mx, my, mz;
    long sy, sz;
    __device__ __forceinline__ long id(int i, int j, int k) const { return (long)i + (long)j * sy + (long)k * sz; }
};

// ---- wall-row fold: f(2) += f(1)/2, f(mz-3) += f(mz-2)/2, rows 0,1,mz-2,mz-1 -> 0 ----
static __global__ void k_adj_fold_rows(Geo<double> g, F8<double> f, int nf) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.mx) return;
    int j = blockIdx.y;
    long b = (long)i + (long)j * g.sy;
    for (int m = 0; m < nf; ++m) {
        double* a = f.f[m];
        a[b + 2 * g.sz] += 0.5 * a[b + 1 * g.sz];
        a[b + (long)(g.mz - 3) * g.sz] += 0.5 * a[b + (long)(g.mz - 2) * g.sz];
        a[b] = 0.0;
        a[b + g.sz] = 0.0;
        a[b + (long)(g.mz - 2) * g.sz] = 0.0;
        a[b + (long)(g.mz - 1) * g.sz] = 0.0;
    }
}

// smoothing coefficient of node (i,j,k) for a kind (0 radial, from the precomputed field cr;
// 1 constant 1/8; 2 x-profile)
__device__ __forceinline__ double adj_coef(const Geo<double>& g, const double* cr, int kind, int i, int j, int k) {
    if (kind == 1) return 0.125;
    if (kind == 2) return g.cbx[i];
    return cr[(long)i + (long)j * g.sy + (long)k * g.sz];
}

// the radial coefficient at every node, once per adjoint call
static __global__ void k_adj_cr(Geo<double> g, double* cr) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.mx) return;
    int j = blockIdx.y, k = blockIdx.z;
    const double xx = g.xc[i], yy = g.yc[j], zz = g.zc[k];
    cr[(long)i + (long)j * g.sy + (long)k * g.sz] = radial_coef(sqrt(xx * xx + yy * yy + zz * zz));
}

// transpose of one smoothing pass.  The input ybar is the adjoint of the pass output with
// its wall rows; folding them (y(1) = y(2)/2 -> ybar(2) += ybar(1)/2, same at the top; rows 0
// and mz-1 constant) is done on the fly.  Then
//   x = y (1 - c sum(wp+wm)) at interior n  +  sum over interior neighbours m of y(m) c(m) w(m->n)
template <int NFLD>
__global__ void k_adj_pass(Geo<double> g, const double* cr, FS<double, NFLD> in, FS<double, NFLD> out, unsigned kinds) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.mx) return;
    int j = blockIdx.y, k = blockIdx.z;
    const int im = wrapi(i - 1, g.mx), ip = wrapi(i + 1, g.mx), jm = wrapi(j - 1, g.my), jp = wrapi(j + 1, g.my);
    const bool intr = k >= 2 && k <= g.mz - 3;
    const bool zm = (k - 1) >= 2 && (k - 1) <= g.mz - 3, zp = (k + 1) >= 2 && (k + 1) <= g.mz - 3;
    const long c = (long)i + (long)j * g.sy + (long)k * g.sz;
    // folded adjoint at node (ii, jj, kk) of an interior row
    auto Y = [&](const double* y, long q, int kk) {
        double v = y[q];
        if (kk == 2) v += 0.5 * y[q - g.sz];
        if (kk == g.mz - 3) v += 0.5 * y[q + g.sz];
        return v;
    };
    // neighbour coefficients, loaded once per kind (the fields of one launch share at most two)
    int lastkind = -1;
    double cn = 0, cxm = 0, cxp = 0, cym = 0, cyp = 0, czm = 0, czp = 0;
#pragma unroll
    for (int q = 0; q < NFLD; ++q) {
        const int kind = (kinds >> (2 * q)) & 3u;
        if (kind != lastkind) {
            lastkind = kind;
            if (intr) {
                cn = adj_coef(g, cr, kind, i, j, k) * (g.wpx[i] + g.wmx[i] + g.wpy[j] + g.wmy[j] + g.wpz[k] + g.wmz[k]);
                cxm = adj_coef(g, cr, kind, im, j, k) * g.wpx[im];
                cxp = adj_coef(g, cr, kind, ip, j, k) * g.wmx[ip];
                cym = adj_coef(g, cr, kind, i, jm, k) * g.wpy[jm];
                cyp = adj_coef(g, cr, kind, i, jp, k) * g.wmy[jp];
            }
            if (zm) czm = adj_coef(g, cr, kind, i, j, k - 1) * g.wpz[k - 1];
            if (zp) czp = adj_coef(g, cr, kind, i, j, k + 1) * g.wmz[k + 1];
        }
        const double* y = in.f[q];
        double v = 0.0;
        if (intr) {
            v += Y(y, c, k) * (1.0 - cn);
            v += Y(y, c - i + im, k) * cxm;
            v += Y(y, c - i + ip, k) * cxp;
            v += Y(y, c + (long)(jm - j) * g.sy, k) * cym;
            v += Y(y, c + (long)(jp - j) * g.sy, k) * cyp;
        }
        if (zm) v += Y(y, c - g.sz, k - 1) * czm;
        if (zp) v += Y(y, c + g.sz, k + 1) * czp;
        out.f[q][c] = v;
    }
}

// (D^T w)(n) along one axis for the first-derivative stencil with per-node coefficients:
//   D f(c) = a_c f(c+1) + (-a+b-c+d)_c f(c) - b_c f(c-1) + c_c f(c+2) - d_c f(c-2)
struct DT {
    __device__ static __forceinline__ double x(const Geo<double>& g, const double* w, int i, int j, int k) {
        const long b = (long)j * g.sy + (long)k * g.sz;
        const int i1 = wrapi(i - 1, g.mx), i2 = wrapi(i - 2, g.mx), p1 = wrapi(i + 1, g.mx), p2 = wrapi(i + 2, g.mx);
        return w[b + i] * (-g.a1x[i] + g.b1x[i] - g.c1x[i] + g.d1x[i]) + w[b + i1] * g.a1x[i1] - w[b + p1] * g.b1x[p1] +
               w[b + i2] * g.c1x[i2] - w[b + p2] * g.d1x[p2];
    }
    __device__ static __forceinline__ double y(const Geo<double>& g, const double* w, int i, int j, int k) {
        const long b = (long)i + (long)k * g.sz;
        const int j1 = wrapi(j - 1, g.my), j2 = wrapi(j - 2, g.my), p1 = wrapi(j + 1, g.my), p2 = wrapi(j + 2, g.my);
        return w[b + j * g.sy] * (-g.a1y[j] + g.b1y[j] - g.c1y[j] + g.d1y[j]) + w[b + j1 * g.sy] * g.a1y[j1] -
               w[b + p1 * g.sy] * g.b1y[p1] + w[b + j2 * g.sy] * g.c1y[j2] - w[b + p2 * g.sy] * g.d1y[p2];
    }
    // w is zero outside the interior rows and the z coefficients are zero there too
    __device__ static __forceinline__ double z(const Geo<double>& g, const double* w, int i, int j, int k) {
        const long b = (long)i + (long)j * g.sy;
        auto W = [&](int kk) { return (kk >= 0 && kk < g.mz) ? w[b + (long)kk * g.sz] : 0.0; };
        auto A = [&](const double* t, int kk) { return (kk >= 0 && kk < g.mz) ? t[kk] : 0.0; };
        return W(k) * (-g.a1z[k] + g.b1z[k] - g.c1z[k] + g.d1z[k]) + W(k - 1) * A(g.a1z, k - 1) - W(k + 1) * A(g.b1z, k + 1) +
               W(k - 2) * A(g.c1z, k - 2) - W(k + 2) * A(g.d1z, k + 2);
    }
};

// out (+)= s * curl^T(w):  curl(B) = (Dy B3 - Dz B2, Dz B1 - Dx B3, Dx B2 - Dy B1), so
//   curl^T(w) = (Dz^T w2 - Dy^T w3, Dx^T w3 - Dz^T w1, Dy^T w1 - Dx^T w2)
static __global__ void k_adj_curlT(Geo<double> g, F3<double> w, F3<double> out, double s, int accumulate) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.mx) return;
    int j = blockIdx.y, k = blockIdx.z;
    long c = (long)i + (long)j * g.sy + (long)k * g.sz;
    double o0 = DT::z(g, w.f[1], i, j, k) - DT::y(g, w.f[2], i, j, k);
    double o1 = DT::x(g, w.f[2], i, j, k) - DT::z(g, w.f[0], i, j, k);
    double o2 = DT::y(g, w.f[0], i, j, k) - DT::x(g, w.f[1], i, j, k);
    if (accumulate) { out.f[0][c] += s * o0; out.f[1][c] += s * o1; out.f[2][c] += s * o2; }
    else { out.f[0][c] = s * o0; out.f[1][c] = s * o1; out.f[2][c] = s * o2; }
}

// Pointwise adjoints at every node, given
//   eb  = adjoint of E0 (all nodes), hb = adjoint of the Hall field H0 (rows folded),
//   ob  = adjoint of the hydro outputs xdif 0,1,2,3,7 (rows folded)
// and the state S (perturbation form) and smoothed current J.  Produces
//   sb  += direct adjoints of rho, m1..3, B1..3, p (8 fields)
//   jb   = adjoint of J (3)
//   wq   = weighted fields for the stencil transposes done by k_adj_gather:
//          0: -di*hb1/rho  1: -di*hb2/rho  2: -di*hb3/rho (Hall grad p)
//          3: ob7*v1  4: ob7*v2  5: ob7*v3 (v . grad p)   6: ob7*gamma*p (gamma p div v)
//   ub   = pointwise adjoint of u_d = m_d/rho at the node from the pressure equation (3)
//   eta  partial sums (one per block)
struct AdjPtw {
    F8<double> s;
    F3<double> j, eb, hb, jb, ub;
    const double* ob[5];
    F8<double> sb, wq;
    double* etapart;
    int hall;
};

static __global__ void k_adj_pointwise(Geo<double> g, AdjPtw a) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y, k = blockIdx.z;
    double eta_acc = 0.0;
    if (i < g.mx) {
        long c = (long)i + (long)j * g.sy + (long)k * g.sz;
        const double rho = g.rho0[k] + a.s.f[0][c];
        const double ri = 1.0 / rho;
        const double m1 = a.s.f[1][c], m2 = a.s.f[2][c], m3 = a.s.f[3][c];
        const double b1 = g.bx0[k] + a.s.f[4][c], b2 = g.by0[k] + a.s.f[5][c], b3 = g.bz0[k] + a.s.f[6][c];
        const double j1 = a.j.f[0][c], j2 = a.j.f[1][c], j3 = a.j.f[2][c];
        double rb = 0, m1b = 0, m2b = 0, m3b = 0, b1b = 0, b2b = 0, b3b = 0, pb = 0, j1b = 0, j2b = 0, j3b = 0;
        // E0 = (-m x B)/rho + eta J
        const double e1 = a.eb.f[0][c], e2 = a.eb.f[1][c], e3 = a.eb.f[2][c];
        {
            const double n1 = -m2 * b3 + m3 * b2, n2 = -m3 * b1 + m1 * b3, n3 = -m1 * b2 + m2 * b1;
            m1b += (b3 * e2 - b2 * e3) * ri;
            m2b += (-b3 * e1 + b1 * e3) * ri;
            m3b += (b2 * e1 - b1 * e2) * ri;
            b1b += (-m3 * e2 + m2 * e3) * ri;
            b2b += (m3 * e1 - m1 * e3) * ri;
            b3b += (-m2 * e1 + m1 * e2) * ri;
            rb += -(n1 * e1 + n2 * e2 + n3 * e3) * ri * ri;
            j1b += g.eta * e1; j2b += g.eta * e2; j3b += g.eta * e3;
            eta_acc += j1 * e1 + j2 * e2 + j3 * e3;
        }
        const bool intr = k >= 2 && k <= g.mz - 3;
        double wq0 = 0, wq1 = 0, wq2 = 0, wq3 = 0, wq4 = 0, wq5 = 0, wq6 = 0, u1 = 0, u2 = 0, u3 = 0;
        if (intr) {
            Nbr<double> n(g, i, j, k);
            if (a.hall) {   // H0 = di (J x B - grad p)/rho
                const double h1 = a.hb.f[0][c], h2 = a.hb.f[1][c], h3 = a.hb.f[2][c];
                const double px = n.Dx(g, a.s.f[7]), py = n.Dy(g, a.s.f[7]), pz = n.Dz(g, a.s.f[7]) + g.dzp0[k];
                const double q1 = j2 * b3 - j3 * b2 - px, q2 = j3 * b1 - j1 * b3 - py, q3 = j1 * b2 - j2 * b1 - pz;
                const double d = g.di * ri;
                j1b += d * (-b3 * h2 + b2 * h3);
                j2b += d * (b3 * h1 - b1 * h3);
                j3b += d * (-b2 * h1 + b1 * h2);
                b1b += d * (j3 * h2 - j2 * h3);
                b2b += d * (-j3 * h1 + j1 * h3);
                b3b += d * (j2 * h1 - j1 * h2);
                rb += -d * ri * (q1 * h1 + q2 * h2 + q3 * h3);
                wq0 = -d * h1; wq1 = -d * h2; wq2 = -d * h3;
            }
            // hydro outputs: J x B in the momentum, the pressure equation
            const double o1 = a.ob[1][c], o2 = a.ob[2][c], o3 = a.ob[3][c], o7 = a.ob[4][c];
            j2b += o1 * b3; j3b -= o1 * b2; b3b += o1 * j2; b2b -= o1 * j3;
            j3b += o2 * b1; j1b -= o2 * b3; b1b += o2 * j3; b3b -= o2 * j1;
            j1b += o3 * b2; j2b -= o3 * b1; b2b += o3 * j1; b1b -= o3 * j2;
            // o7 = -(px v1 + py v2 + pz v3) + gamma p divv + (gamma-1) eta |J|^2
            const double v1 = m1 * ri, v2 = m2 * ri, v3 = m3 * ri;
            const double px = n.Dx(g, a.s.f[7]), py = n.Dy(g, a.s.f[7]), pz = n.Dz(g, a.s.f[7]) + g.dzp0[k];
            auto U = [&](const double* m, long q, int kk) { return m[q] / (g.rho0[kk] + a.s.f[0][q]); };
            const double* M1 = a.s.f[1];
            const double* M2 = a.s.f[2];
            const double* M3 = a.s.f[3];
            const double du1 = d1fc(U(M1, n.xm2, k), U(M1, n.xm1, k), U(M1, n.c, k), U(M1, n.xp1, k), U(M1, n.xp2, k),
                                    g.a1x[i], g.b1x[i], g.c1x[i], g.d1x[i]);
            const double du2 = d1fc(U(M2, n.ym2, k), U(M2, n.ym1, k), U(M2, n.c, k), U(M2, n.yp1, k), U(M2, n.yp2, k),
                                    g.a1y[j], g.b1y[j], g.c1y[j], g.d1y[j]);
            const double du3 = d1fc(U(M3, c - 2 * g.sz, k - 2), U(M3, c - g.sz, k - 1), U(M3, c, k), U(M3, c + g.sz, k + 1),
                                    U(M3, c + 2 * g.sz, k + 2), g.a1z[k], g.b1z[k], g.c1z[k], g.d1z[k]);
            const double divv = -du1 - du2 - du3;
            const double p = g.p0[k] + a.s.f[7][c];
            u1 = -o7 * px; u2 = -o7 * py; u3 = -o7 * pz;   // adjoint of the centre velocity
            pb += o7 * g.gamma * divv;
            wq3 = o7 * v1; wq4 = o7 * v2; wq5 = o7 * v3;
            wq6 = o7 * g.gamma * p;
            const double ce = (g.gamma - 1.0) * g.eta;
            j1b += o7 * 2.0 * ce * j1; j2b += o7 * 2.0 * ce * j2; j3b += o7 * 2.0 * ce * j3;
            eta_acc += o7 * (g.gamma - 1.0) * (j1 * j1 + j2 * j2 + j3 * j3);
        }
        a.sb.f[0][c] += rb; a.sb.f[1][c] += m1b; a.sb.f[2][c] += m2b; a.sb.f[3][c] += m3b;
        a.sb.f[4][c] += b1b; a.sb.f[5][c] += b2b; a.sb.f[6][c] += b3b; a.sb.f[7][c] += pb;
        a.jb.f[0][c] = j1b; a.jb.f[1][c] = j2b; a.jb.f[2][c] = j3b;
        a.wq.f[0][c] = wq0; a.wq.f[1][c] = wq1; a.wq.f[2][c] = wq2; a.wq.f[3][c] = wq3;
        a.wq.f[4][c] = wq4; a.wq.f[5][c] = wq5; a.wq.f[6][c] = wq6;
        a.ub.f[0][c] = u1; a.ub.f[1][c] = u2; a.ub.f[2][c] = u3;
    }
    // block partial of d/d eta
    __shared__ double sh[32];
    double v = warp_sum(eta_acc);
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        int nw = (blockDim.x + 31) >> 5;
        double t = 0;
        for (int w2 = 0; w2 < nw; ++w2) t += sh[w2];
        a.etapart[(long)blockIdx.z * gridDim.y * gridDim.x + (long)blockIdx.y * gridDim.x + blockIdx.x] = t;
    }
}

// Gather of the stencil transposes of the hydro and Hall adjoints, then the pointwise chain
// rule through the fluxes m_d m_k / rho (+ dp on the diagonal), u_d = m_d/rho and p.
//   ob: adjoints of xdif 0,1,2,3,7 (rows folded);  wq, ub from k_adj_pointwise
struct AdjGat {
    F8<double> s, sb, wq;
    F3<double> ub;
    const double* ob[5];
};

static __global__ void k_adj_gather(Geo<double> g, AdjGat a) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.mx) return;
    int j = blockIdx.y, k = blockIdx.z;
    long c = (long)i + (long)j * g.sy + (long)k * g.sz;
    const double rho = g.rho0[k] + a.s.f[0][c];
    const double ri = 1.0 / rho;
    const double m[3] = {a.s.f[1][c], a.s.f[2][c], a.s.f[3][c]};
    // flux adjoints abar[d][q] = -(D_d^T ob_q)(n), q = 0 continuity, 1..3 momentum
    double ab[3][4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        ab[0][q] = -DT::x(g, a.ob[q], i, j, k);
        ab[1][q] = -DT::y(g, a.ob[q], i, j, k);
        ab[2][q] = -DT::z(g, a.ob[q], i, j, k);
    }
    // pressure: dp gets sum_d ab[d][1+d] (flux diagonal) - sum_d D_d^T(ob7 v_d) (v.grad p)
    //           - D^T of the Hall weights; u_d gets -D_d^T(ob7 gamma p) plus the centre term
    double pb = ab[0][1] + ab[1][2] + ab[2][3];
    pb += -DT::x(g, a.wq.f[3], i, j, k) - DT::y(g, a.wq.f[4], i, j, k) - DT::z(g, a.wq.f[5], i, j, k);
    pb += DT::x(g, a.wq.f[0], i, j, k) + DT::y(g, a.wq.f[1], i, j, k) + DT::z(g, a.wq.f[2], i, j, k);
    double ub[3];
    ub[0] = -DT::x(g, a.wq.f[6], i, j, k) + a.ub.f[0][c];
    ub[1] = -DT::y(g, a.wq.f[6], i, j, k) + a.ub.f[1][c];
    ub[2] = -DT::z(g, a.wq.f[6], i, j, k) + a.ub.f[2][c];
    double mb[3] = {0, 0, 0}, rb = 0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        mb[d] += ab[d][0];
#pragma unroll
        for (int q = 1; q <= 3; ++q) {
            // flux m_d m_q / rho
            mb[d] += ab[d][q] * m[q - 1] * ri;
            mb[q - 1] += ab[d][q] * m[d] * ri;
            rb -= ab[d][q] * m[d] * m[q - 1] * ri * ri;
        }
        mb[d] += ub[d] * ri;
        rb -= ub[d] * m[d] * ri * ri;
    }
    a.sb.f[0][c] += rb;
    a.sb.f[1][c] += mb[0];
    a.sb.f[2][c] += mb[1];
    a.sb.f[3][c] += mb[2];
    a.sb.f[7][c] += pb;
}

// *acc += sum(part[0..n)), one block, fixed order
static __global__ void k_reduce_add(const double* part, long n, double* acc) {
    double v = 0.0;
    for (long q = threadIdx.x; q < n; q += blockDim.x) v += part[q];
    __shared__ double sh[32];
    v = warp_sum(v);
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)((blockDim.x + 31) >> 5); ++w) t += sh[w];
        *acc += t;
    }
}

// y = a*x + b*y over 8 fields (vector algebra of the RK adjoint)
static __global__ void k_axpby8(long n, F8<double> y, double b, F8<double> x, double a) {
    long c = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
#pragma unroll
    for (int m = 0; m < 8; ++m) y.f[m][c] = a * x.f[m][c] + b * y.f[m][c];
}

// objective: Phi = (1/my) sum_j sum_i sqrt(Bz(z=0)^2 + eps^2) w_i -> its gradient in Bz
static __global__ void k_adj_flux_seed(Geo<double> g, const double* dbz, const double* wx, double* lam_bz) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.mx) return;
    int j = blockIdx.y;
    if (g.mz % 2) {
        int kc = (g.mz - 1) / 2;
        long c = (long)i + (long)j * g.sy + (long)kc * g.sz;
        double bz = g.bz0[kc] + dbz[c];
        lam_bz[c] = wx[i] * bz / sqrt(bz * bz + 1e-20) / g.my;
    } else {
        int ka = g.mz / 2 - 1, kb = g.mz / 2;
        long ca = (long)i + (long)j * g.sy + (long)ka * g.sz, cb = (long)i + (long)j * g.sy + (long)kb * g.sz;
        double bz = 0.5 * ((g.bz0[ka] + dbz[ca]) + (g.bz0[kb] + dbz[cb]));
        double d = wx[i] * bz / sqrt(bz * bz + 1e-20) / g.my * 0.5;
        lam_bz[ca] = d;
        lam_bz[cb] = d;
    }
}

// psi map transpose: dPhi/dpsi(i,k) = sum_j [ -(Dz^T lam_Bx)(i,j,k) + (Dx^T lam_Bz)(i,j,k) ]
static __global__ void k_adj_psi(Geo<double> g, const double* lbx, const double* lbz, double* out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.mx) return;
    int k = blockIdx.y;
    double s = 0.0;
    for (int j = 0; j < g.my; ++j) s += -DT::z(g, lbx, i, j, k) + DT::x(g, lbz, i, j, k);
    out[(long)i + (long)k * g.mx] = s;
}

// forward psi map: dBx = -Dz psi (interior rows), dBz = Dx psi, added to the state
static __global__ void k_psi_apply(Geo<double> g, const double* psi, double* bx, double* bz, double s) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.mx) return;
    int j = blockIdx.y, k = blockIdx.z;
    long c = (long)i + (long)j * g.sy + (long)k * g.sz;
    const double* P = psi;
    auto ps = [&](int ii, int kk) { return P[(long)wrapi(ii, g.mx) + (long)kk * g.mx]; };
    double dz = 0.0;
    if (k >= 2 && k <= g.mz - 3)
        dz = d1fc(ps(i, k - 2), ps(i, k - 1), ps(i, k), ps(i, k + 1), ps(i, k + 2), g.a1z[k], g.b1z[k], g.c1z[k], g.d1z[k]);
    double dx = d1fc(ps(i - 2, k), ps(i - 1, k), ps(i, k), ps(i + 1, k), ps(i + 2, k), g.a1x[i], g.b1x[i], g.c1x[i], g.d1x[i]);
    bx[c] += s * (-dz);
    bz[c] += s * dx;
}

}  // namespace dasha
