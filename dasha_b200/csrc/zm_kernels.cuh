// zm_kernels.cuh -- z-marching (2.5-D) kernels: each CTA owns an x-y tile of TX x TY
// columns and streams through a chunk of z planes, keeping the planes a stencil needs in
// shared-memory rings.  Global memory is read once per plane (plus the x-y halo, which
// neighbouring CTAs read at about the same time and so mostly hits L2) and written once.
//
// k_zsmooth: P Jacobi smoothing passes of NF fields in one launch.  Level 0 is the source
//   (loaded, or computed pointwise, on the tile plus a P-node halo), level l = pass l on the
//   tile plus P-l, each level one plane behind the previous one.  The wall rows are applied
//   after every pass as in the reference (outer row 0, next row half of its inner neighbour;
//   bndry* t3dsdsc.f:1821-1857 and its copies), so each level's rows 0,1 and mz-2,mz-1 are
//   derived when its rows 2 and mz-3 are computed.  The last level goes to an epilogue: a
//   store, an accumulate, or the RK4 stage update.
// k_rhs_zm: the right-hand side (right, t3dsdsc.f:1334-1566) from a ring of the quantities
//   that are differentiated (6 plane slots: the 5-plane stencil plus the plane being loaded),
//   with the pointwise inputs read at the output node.
// k_zpass: one smoothing pass, z-marching with a register queue for the z neighbours and one
//   shared-memory plane (tile plus a 1-node halo) for the x and y neighbours.
#pragma once
#include "mhd_kernels.cuh"

namespace dasha {

__device__ __forceinline__ int pmod(int i, int n) {
    int r = i % n;
    return r < 0 ? r + n : r;
}

// radial smoothing coefficient 1/32 + (1/8 - 1/32) (1 + tanh((r-3)/3))/2 (t3dsdsc.f:5659-5661)
__device__ __forceinline__ float radial_coef(float r) {
    return 1.0f / 32.0f + (1.0f / 8.0f - 1.0f / 32.0f) * 0.5f * (1.0f + tanhf((r - 3.0f) / 3.0f));
}
__device__ __forceinline__ double radial_coef(double r) {
    return 1.0 / 32.0 + (1.0 / 8.0 - 1.0 / 32.0) * 0.5 * (1 + tanh((r - 3.) / 3.));
}

// ---------------------------------------------------------------------------------------
// sources of k_zsmooth (level 0 at one node)
template <class T, int NF>
struct SrcFields {
    const T* f[NF];
    __device__ __forceinline__ void load(const Geo<T>&, long idx, int, T v[NF]) const {
#pragma unroll
        for (int q = 0; q < NF; ++q) v[q] = f[q][idx];
    }
};

// E = -v x B + eta J at the node (t3dsdsc.f:1367-1372): the k_efield source fused in
template <class T>
struct SrcEfield {
    const T *r, *m1, *m2, *m3, *b1, *b2, *b3, *j1, *j2, *j3;
    __device__ __forceinline__ void load(const Geo<T>& g, long idx, int k, T v[3]) const {
        T rr = T(g.rho0[k]) + r[idx];
        T a1 = m1[idx], a2 = m2[idx], a3 = m3[idx];
        T c1 = T(g.bx0[k]) + b1[idx], c2 = T(g.by0[k]) + b2[idx], c3 = T(g.bz0[k]) + b3[idx];
        v[0] = (-a2 * c3 + a3 * c2) / rr + g.eta * j1[idx];
        v[1] = (-a3 * c1 + a1 * c3) / rr + g.eta * j2[idx];
        v[2] = (-a1 * c2 + a2 * c1) / rr + g.eta * j3[idx];
    }
};

// ---------------------------------------------------------------------------------------
// epilogues of k_zsmooth (last level at one node, every plane including the wall rows)
// Every epilogue has a register payload Pre filled by pre(idx) one plane ahead of
// store(idx, v, pre), so that its global loads overlap the plane's barrier and stencil.
template <class T, int NF>
struct EpiStore {
    T* f[NF];
    struct Pre {};
    __device__ __forceinline__ void pre(long, Pre&) const {}
    __device__ __forceinline__ void store(const Geo<T>& g, long idx, const T v[NF], const Pre&) const { store(g, idx, v); }
    __device__ __forceinline__ void store(const Geo<T>&, long idx, const T v[NF]) const {
#pragma unroll
        for (int q = 0; q < NF; ++q) f[q][idx] = v[q];
    }
};

template <class T, int NF>
struct EpiAcc {   // f = a + v   (a may alias f: each node is read and written by one thread)
    T* f[NF];
    const T* a[NF];
    struct Pre { T a[NF]; };
    __device__ __forceinline__ void pre(long idx, Pre& p) const {
#pragma unroll
        for (int q = 0; q < NF; ++q) p.a[q] = a[q][idx];
    }
    __device__ __forceinline__ void store(const Geo<T>&, long idx, const T v[NF], const Pre& p) const {
#pragma unroll
        for (int q = 0; q < NF; ++q) f[q][idx] = p.a[q] + v[q];
    }
    __device__ __forceinline__ void store(const Geo<T>&, long idx, const T v[NF]) const {
#pragma unroll
        for (int q = 0; q < NF; ++q) f[q][idx] = a[q][idx] + v[q];
    }
};

// Post-step filter on a compensated FP32 state (x, comp), exact value x - comp: the filter's
// increment v is added with a Kahan step, and the wall rows of the result are set to the exact
// halves / zeros of row 2 and row mz-3 (bndrytt), so the filter loses no more than the
// increment's own rounding.
template <class T, int NF>
struct EpiKF {
    T* x[NF];
    T* comp[NF];
    struct Pre { T x[NF], k[NF]; };
    __device__ __forceinline__ void pre(long idx, Pre& p) const {
#pragma unroll
        for (int q = 0; q < NF; ++q) { p.x[q] = x[q][idx]; p.k[q] = comp[q][idx]; }
    }
    // interior node idx; when wall, also the wall-adjacent row ih (half) and the wall row iz (0)
    __device__ __forceinline__ void store_rows(long idx, bool wall, long ih, long iz, const T v[NF],
                                               const Pre& p) const {
#pragma unroll
        for (int q = 0; q < NF; ++q) {
            const T y = v[q] - p.k[q];
            const T t = p.x[q] + y;
            const T kk = (t - p.x[q]) - y;
            x[q][idx] = t;
            comp[q][idx] = kk;
            if (wall) {
                x[q][ih] = T(0.5) * t; comp[q][ih] = T(0.5) * kk;
                x[q][iz] = T(0); comp[q][iz] = T(0);
            }
        }
    }
};

// RK4 stage update with the smoothed xdif (stepon t3dsdsc.f:1090-1132), same arithmetic as
// k_rk: plain registers (base, acc = xm, x) in FP64, increment-only acc plus a Kahan base
// update in FP32.
template <class T, int NF, bool KAHAN>
struct EpiRK {
    T* x[NF];
    const T* base[NF];
    T* acc[NF];
    T* comp[NF];
    int stage;
    double dt;
    struct Pre { T b[NF], a[NF], k[NF]; };
    __device__ __forceinline__ void pre(long c, Pre& p) const {
#pragma unroll
        for (int m = 0; m < NF; ++m) {
            p.b[m] = (stage == 4 && !KAHAN) ? T(0) : base[m][c];
            p.a[m] = stage == 1 ? T(0) : acc[m][c];
            p.k[m] = (KAHAN && stage == 4) ? comp[m][c] : T(0);
        }
    }
    __device__ __forceinline__ void store(const Geo<T>&, long c, const T v[NF], const Pre& p) const {
        const T tdt = T(dt);
#pragma unroll
        for (int m = 0; m < NF; ++m) {
            const T kv = v[m], b = p.b[m];
            if (!KAHAN) {
                if (stage == 1) { acc[m][c] = b + kv * tdt / T(6.); x[m][c] = b + kv * tdt / T(2.); }
                else if (stage == 2) { acc[m][c] = p.a[m] + kv * tdt / T(3.); x[m][c] = b + kv * tdt / T(2.); }
                else if (stage == 3) { acc[m][c] = p.a[m] + kv * tdt / T(3.); x[m][c] = b + kv * tdt; }
                else { x[m][c] = p.a[m] + kv * tdt / T(6.); }
            } else {
                if (stage == 1) { acc[m][c] = kv * tdt / T(6.); x[m][c] = b + kv * tdt / T(2.); }
                else if (stage == 2) { acc[m][c] = p.a[m] + kv * tdt / T(3.); x[m][c] = b + kv * tdt / T(2.); }
                else if (stage == 3) { acc[m][c] = p.a[m] + kv * tdt / T(3.); x[m][c] = b + kv * tdt; }
                else {
                    const T inc = p.a[m] + kv * tdt / T(6.);
                    const T y = inc - p.k[m];
                    const T t = b + y;
                    comp[m][c] = (t - b) - y;
                    x[m][c] = t;
                }
            }
        }
    }
    __device__ __forceinline__ void store(const Geo<T>&, long c, const T v[NF]) const {
        const T tdt = T(dt);
#pragma unroll
        for (int m = 0; m < NF; ++m) {
            T kv = v[m];
            T b = base[m][c];
            if (!KAHAN) {
                if (stage == 1) { acc[m][c] = b + kv * tdt / T(6.); x[m][c] = b + kv * tdt / T(2.); }
                else if (stage == 2) { acc[m][c] = acc[m][c] + kv * tdt / T(3.); x[m][c] = b + kv * tdt / T(2.); }
                else if (stage == 3) { acc[m][c] = acc[m][c] + kv * tdt / T(3.); x[m][c] = b + kv * tdt; }
                else { x[m][c] = acc[m][c] + kv * tdt / T(6.); }
            } else {
                if (stage == 1) { acc[m][c] = kv * tdt / T(6.); x[m][c] = b + kv * tdt / T(2.); }
                else if (stage == 2) { acc[m][c] = acc[m][c] + kv * tdt / T(3.); x[m][c] = b + kv * tdt / T(2.); }
                else if (stage == 3) { acc[m][c] = acc[m][c] + kv * tdt / T(3.); x[m][c] = b + kv * tdt; }
                else {
                    T inc = acc[m][c] + kv * tdt / T(6.);
                    T y = inc - comp[m][c];
                    T t = b + y;
                    comp[m][c] = (t - b) - y;
                    x[m][c] = t;
                }
            }
        }
    }
};

// ---------------------------------------------------------------------------------------
template <int TX, int TY, int P>
struct ZReg {
    __host__ __device__ static constexpr int W(int l) { return TX + 2 * (P - l); }
    __host__ __device__ static constexpr int H(int l) { return TY + 2 * (P - l); }
    __host__ __device__ static constexpr int S(int l) { return W(l) * H(l); }
    // ring of level l: 4 plane slots x NF fields x S(l)
    __host__ __device__ static constexpr long off(int l, int nf) {
        long o = 0;
        for (int m = 0; m < l; ++m) o += 4L * nf * S(m);
        return o;
    }
    __host__ __device__ static constexpr long total(int nf) { return off(P, nf); }
};

template <class T, int NF, int P, int TX, int TY>
constexpr size_t zsmooth_smem_bytes() {
    return sizeof(T) * ZReg<TX, TY, P>::total(NF);
}

// kinds: 2 bits per field, 0 radial coefficient, 1 constant 1/8, 2 x-profile (B in avrg)
template <class T, int NF, int P, int TX, int TY, class Src, class Epi>
__global__ void __launch_bounds__(TX* TY) k_zsmooth(Geo<T> g, Src src, Epi epi, unsigned kinds, int chunk) {
    using R = ZReg<TX, TY, P>;
    constexpr int NT = TX * TY;
    constexpr int S0 = R::S(0);
    constexpr int NPF = (S0 + NT - 1) / NT;
    extern __shared__ __align__(16) unsigned char zs_smem_raw[];
    T* sm = reinterpret_cast<T*>(zs_smem_raw);

    const int tid = threadIdx.x;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const int mz = g.mz;
    const int k0 = blockIdx.z * chunk;
    const int k1 = min(k0 + chunk, mz);   // outputs of this CTA: planes [k0, k1)
    bool need_r = false;
#pragma unroll
    for (int q = 0; q < NF; ++q) need_r |= ((kinds >> (2 * q)) & 3u) == 0u;

    // prefetch registers for level-0 planes
    T pre[NPF][NF];
    auto issue = [&](int t) {
#pragma unroll
        for (int u = 0; u < NPF; ++u) {
            int q = tid + u * NT;
            if (q < S0) {
                int li = q % R::W(0), lj = q / R::W(0);
                int gi = pmod(x0 - P + li, g.mx), gj = pmod(y0 - P + lj, g.my);
                src.load(g, (long)gi + (long)gj * g.sy + (long)t * g.sz, t, pre[u]);
            }
        }
    };
    const int tA = k0 - P, tB = k1 - 1 + P;
    if (tA >= 0 && tA < mz) issue(tA);
    else if (tA < 0 && 0 <= tB) issue(0);   // first valid plane is 0
    for (int t = tA; t <= tB; ++t) {
        if (t >= 0 && t < mz) {
            T* r0 = sm + R::off(0, NF) + (long)(t & 3) * NF * S0;
#pragma unroll
            for (int u = 0; u < NPF; ++u) {
                int q = tid + u * NT;
                if (q < S0) {
#pragma unroll
                    for (int f = 0; f < NF; ++f) r0[f * S0 + q] = pre[u][f];
                }
            }
        }
        __syncthreads();
        if (t + 1 >= 0 && t + 1 < mz && t + 1 <= tB) issue(t + 1);
#pragma unroll
        for (int l = 1; l <= P; ++l) {
            const int c = t - l;
            const int halo = P - l;
            const bool active = c >= 2 && c <= mz - 3 && c >= k0 - halo && c <= k1 - 1 + halo;
            if (active) {
                const int Wl = R::W(l), Sl = R::S(l);
                const int Wp = R::W(l - 1), Sp = R::S(l - 1);
                const T* rin = sm + R::off(l - 1, NF);
                const T* pc = rin + (long)(c & 3) * NF * Sp;
                const T* pm = rin + (long)((c - 1) & 3) * NF * Sp;
                const T* pp = rin + (long)((c + 1) & 3) * NF * Sp;
                const T wpz = g.wpz[c], wmz = g.wmz[c], zc = g.zc[c];
                for (int q = tid; q < Sl; q += NT) {
                    const int li = q % Wl, lj = q / Wl;
                    const int xi = x0 - halo + li, yj = y0 - halo + lj;
                    const int gi = pmod(xi, g.mx), gj = pmod(yj, g.my);
                    const int qi = (lj + 1) * Wp + (li + 1);
                    const T wpx = g.wpx[gi], wmx = g.wmx[gi], wpy = g.wpy[gj], wmy = g.wmy[gj];
                    T cr = T(0);
                    if (need_r) {
                        const T xx = g.xc[gi], yy = g.yc[gj];
                        cr = radial_coef(sqrt(xx * xx + yy * yy + zc * zc));
                    }
                    T val[NF];
#pragma unroll
                    for (int f = 0; f < NF; ++f) {
                        const T* a = pc + f * Sp;
                        const T f0 = a[qi];
                        const T tx = (a[qi + 1] - f0) * wpx - (f0 - a[qi - 1]) * wmx;
                        const T ty = (a[qi + Wp] - f0) * wpy - (f0 - a[qi - Wp]) * wmy;
                        const T tz = (pp[f * Sp + qi] - f0) * wpz - (f0 - pm[f * Sp + qi]) * wmz;
                        const unsigned kind = (kinds >> (2 * f)) & 3u;
                        const T coef = kind == 0u ? cr : (kind == 1u ? T(0.125) : g.cbx[gi]);
                        val[f] = f0 + coef * (tx + ty + tz);
                    }
                    if (l < P) {
                        T* ro = sm + R::off(l, NF);
#pragma unroll
                        for (int f = 0; f < NF; ++f) {
                            ro[(long)(c & 3) * NF * Sl + f * Sl + q] = val[f];
                            if (c == 2) {
                                ro[1L * NF * Sl + f * Sl + q] = T(0.5) * val[f];
                                ro[0L * NF * Sl + f * Sl + q] = T(0);
                            }
                            if (c == mz - 3) ro[(long)((mz - 2) & 3) * NF * Sl + f * Sl + q] = T(0.5) * val[f];
                        }
                    } else if (xi < g.mx && yj < g.my) {
                        const long base = (long)xi + (long)yj * g.sy;
                        epi.store(g, base + (long)c * g.sz, val);
                        if (c == 2 || c == mz - 3) {
                            T hv[NF], zv[NF];
#pragma unroll
                            for (int f = 0; f < NF; ++f) { hv[f] = T(0.5) * val[f]; zv[f] = T(0); }
                            const int kh = c == 2 ? 1 : mz - 2, kz = c == 2 ? 0 : mz - 1;
                            epi.store(g, base + (long)kh * g.sz, hv);
                            epi.store(g, base + (long)kz * g.sz, zv);
                        }
                    }
                }
            }
            if (l < P) __syncthreads();
        }
    }
}

// ---------------------------------------------------------------------------------------
// Right-hand side, z-marching.  Ring quantities (6 plane slots, tile + 2 halo):
//   0 rinv = 1/rho   1 m1   2 m2   3 m3   4 dp (p - p0)   5 E1   6 E2   7 E3   8 drho
constexpr int RQ = 9;

template <int TX, int TY>
struct RReg {
    static constexpr int W = TX + 4, H = TY + 4, S = W * H;
};

template <class T, int TX, int TY>
constexpr size_t rhs_smem_bytes() {
    return sizeof(T) * 6L * RQ * RReg<TX, TY>::S;
}

template <class T, int TX, int TY>
__global__ void __launch_bounds__(TX* TY) k_rhs_zm(Geo<T> g, F8<T> x, F3<T> cur, F3<T> e, F8<T> xdif, int chunk) {
    using R = RReg<TX, TY>;
    constexpr int NT = TX * TY;
    constexpr int S = R::S, W = R::W;
    constexpr int NPF = (S + NT - 1) / NT;
    extern __shared__ __align__(16) unsigned char rz_smem_raw[];
    T* sm = reinterpret_cast<T*>(rz_smem_raw);
    const int tid = threadIdx.x;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const int mz = g.mz;
    const int k0 = blockIdx.z * chunk;
    const int k1 = min(k0 + chunk, mz);

    T pre[NPF][RQ];
    auto issue = [&](int t) {
        const T r0 = T(g.rho0[t]);
#pragma unroll
        for (int u = 0; u < NPF; ++u) {
            int q = tid + u * NT;
            if (q < S) {
                int li = q % W, lj = q / W;
                int gi = pmod(x0 - 2 + li, g.mx), gj = pmod(y0 - 2 + lj, g.my);
                long idx = (long)gi + (long)gj * g.sy + (long)t * g.sz;
                T dr = x.f[0][idx];
                pre[u][0] = T(1) / (r0 + dr);
                pre[u][1] = x.f[1][idx];
                pre[u][2] = x.f[2][idx];
                pre[u][3] = x.f[3][idx];
                pre[u][4] = x.f[7][idx];
                pre[u][5] = e.f[0][idx];
                pre[u][6] = e.f[1][idx];
                pre[u][7] = e.f[2][idx];
                pre[u][8] = dr;
            }
        }
    };
    const int tA = max(k0 - 2, 0), tB = min(k1 + 1, mz - 1);
    issue(tA);
    // per-column coefficients and the pointwise inputs of the output node, one plane ahead
    const int li = tid % TX, lj = tid / TX;
    const int xi = x0 + li, yj = y0 + lj;
    const bool out_ok = xi < g.mx && yj < g.my;
    const int i = out_ok ? xi : 0, jj = out_ok ? yj : 0;
    const T ax = g.a1x[i], bx = g.b1x[i], cx = g.c1x[i], dx = g.d1x[i];
    const T ay = g.a1y[jj], by = g.b1y[jj], cy = g.c1y[jj], dy = g.d1y[jj];
    struct PW { T b1, b2, b3, j1, j2, j3, az, bz, cz, dz, rsx, rsy, rsz, dzp0, p0; };
    auto loadpw = [&](int c, PW& w) {
        const long ci = (long)i + (long)jj * g.sy + (long)c * g.sz;
        w.b1 = T(g.bx0[c]) + x.f[4][ci]; w.b2 = T(g.by0[c]) + x.f[5][ci]; w.b3 = T(g.bz0[c]) + x.f[6][ci];
        w.j1 = cur.f[0][ci]; w.j2 = cur.f[1][ci]; w.j3 = cur.f[2][ci];
        w.az = g.a1z[c]; w.bz = g.b1z[c]; w.cz = g.c1z[c]; w.dz = g.d1z[c];
        w.rsx = T(g.rsx[c]); w.rsy = T(g.rsy[c]); w.rsz = T(g.rsz[c]); w.dzp0 = T(g.dzp0[c]); w.p0 = T(g.p0[c]);
    };
    PW npw;
    const int cfirst = max(k0, 2);
    if (cfirst <= min(k1 - 1, mz - 3)) loadpw(cfirst, npw);
    for (int t = tA; t <= tB; ++t) {
        {
            T* r0 = sm + (long)(t % 6) * RQ * S;
#pragma unroll
            for (int u = 0; u < NPF; ++u) {
                int q = tid + u * NT;
                if (q < S) {
#pragma unroll
                    for (int f = 0; f < RQ; ++f) r0[f * S + q] = pre[u][f];
                }
            }
        }
        __syncthreads();
        if (t + 1 <= tB) issue(t + 1);
        const int c = t - 2;
        if (c >= 2 && c <= mz - 3 && c >= k0 && c < k1) {
            const PW pw = npw;
            if (c + 1 <= min(k1 - 1, mz - 3)) loadpw(c + 1, npw);
            if (out_ok) {
                const int q = (lj + 2) * W + (li + 2);
                const T* Z[5];
#pragma unroll
                for (int s = 0; s < 5; ++s) Z[s] = sm + (long)((c - 2 + s) % 6) * RQ * S;
                const T* C0 = Z[2];
                auto X = [&](int f, int s) { return C0[f * S + q + (s - 2)]; };        // x-neighbours
                auto Y = [&](int f, int s) { return C0[f * S + q + (s - 2) * W]; };    // y-neighbours
                auto Zz = [&](int f, int s) { return Z[s][f * S + q]; };             // z-neighbours
                const T az = pw.az, bz = pw.bz, cz = pw.cz, dz = pw.dz;
                auto DX = [&](auto fn) { return d1fc(fn(0), fn(1), fn(2), fn(3), fn(4), ax, bx, cx, dx); };
                auto DY = [&](auto fn) { return d1fc(fn(0), fn(1), fn(2), fn(3), fn(4), ay, by, cy, dy); };
                auto DZ = [&](auto fn) { return d1fc(fn(0), fn(1), fn(2), fn(3), fn(4), az, bz, cz, dz); };
                T out[NF];
                // continuity
                out[0] = -DX([&](int s) { return X(1, s); }) - DY([&](int s) { return Y(2, s); }) -
                         DZ([&](int s) { return Zz(3, s); });
                // momentum fluxes (flux, t3dsdsc.f:2317-2347)
                out[1] = -DX([&](int s) { return X(1, s) * X(1, s) * X(0, s) + X(4, s); }) -
                         DY([&](int s) { return Y(1, s) * Y(2, s) * Y(0, s); }) -
                         DZ([&](int s) { return Zz(1, s) * Zz(3, s) * Zz(0, s); });
                out[2] = -DX([&](int s) { return X(1, s) * X(2, s) * X(0, s); }) -
                         DY([&](int s) { return Y(2, s) * Y(2, s) * Y(0, s) + Y(4, s); }) -
                         DZ([&](int s) { return Zz(2, s) * Zz(3, s) * Zz(0, s); });
                out[3] = -DX([&](int s) { return X(1, s) * X(3, s) * X(0, s); }) -
                         DY([&](int s) { return Y(2, s) * Y(3, s) * Y(0, s); }) -
                         DZ([&](int s) { return Zz(3, s) * Zz(3, s) * Zz(0, s) + Zz(4, s); });
                const long cidx = (long)i + (long)jj * g.sy + (long)c * g.sz;
                const T b1 = pw.b1, b2 = pw.b2, b3 = pw.b3;
                const T j1 = pw.j1, j2 = pw.j2, j3 = pw.j3;
                out[1] = out[1] - pw.rsx + j2 * b3 - j3 * b2;
                out[2] = out[2] - pw.rsy + j3 * b1 - j1 * b3;
                out[3] = out[3] - pw.rsz + j1 * b2 - j2 * b1;
                // induction
                out[4] = -DY([&](int s) { return Y(7, s); }) + DZ([&](int s) { return Zz(6, s); });
                out[5] = -DZ([&](int s) { return Zz(5, s); }) + DX([&](int s) { return X(7, s); });
                out[6] = -DX([&](int s) { return X(6, s); }) + DY([&](int s) { return Y(5, s); });
                // pressure
                const T ri = X(0, 2);
                const T v1 = X(1, 2) * ri, v2 = X(2, 2) * ri, v3 = X(3, 2) * ri;
                const T px = DX([&](int s) { return X(4, s); });
                const T py = DY([&](int s) { return Y(4, s); });
                const T pz = DZ([&](int s) { return Zz(4, s); }) + pw.dzp0;
                const T divv = -DX([&](int s) { return X(1, s) * X(0, s); }) - DY([&](int s) { return Y(2, s) * Y(0, s); }) -
                               DZ([&](int s) { return Zz(3, s) * Zz(0, s); });
                const T pc = pw.p0 + X(4, 2);
                out[7] = -px * v1 - py * v2 - pz * v3 + divv * g.gamma * pc +
                         (g.gamma - T(1)) * g.eta * (j1 * j1 + j2 * j2 + j3 * j3);
                if (g.viscos) {
                    const T a2x = g.a2x[i], b2x = g.b2x[i], c2x = g.c2x[i], d2x = g.d2x[i];
                    const T a2y = g.a2y[jj], b2y = g.b2y[jj], c2y = g.c2y[jj], d2y = g.d2y[jj];
                    const T a2z = g.a2z[c], b2z = g.b2z[c], c2z = g.c2z[c], d2z = g.d2z[c];
                    auto L = [&](int f) {
                        return d1fc(X(f, 0) * X(0, 0), X(f, 1) * X(0, 1), X(f, 2) * X(0, 2), X(f, 3) * X(0, 3),
                                    X(f, 4) * X(0, 4), a2x, b2x, c2x, d2x) +
                               d1fc(Y(f, 0) * Y(0, 0), Y(f, 1) * Y(0, 1), Y(f, 2) * Y(0, 2), Y(f, 3) * Y(0, 3),
                                    Y(f, 4) * Y(0, 4), a2y, b2y, c2y, d2y) +
                               d1fc(Zz(f, 0) * Zz(0, 0), Zz(f, 1) * Zz(0, 1), Zz(f, 2) * Zz(0, 2),
                                    Zz(f, 3) * Zz(0, 3), Zz(f, 4) * Zz(0, 4), a2z, b2z, c2z, d2z);
                    };
                    const T af = L(1), ag = L(2), ah = L(3);
                    out[1] = out[1] + g.mu * af;
                    out[2] = out[2] + g.mu * ag;
                    out[3] = out[3] + g.mu * ah;
                    out[7] = out[7] + g.mu * (v1 * af + v2 * ag + v3 * ah);
                }
                if (g.diffu) {
                    const T a2x = g.a2x[i], b2x = g.b2x[i], c2x = g.c2x[i], d2x = g.d2x[i];
                    const T a2y = g.a2y[jj], b2y = g.b2y[jj], c2y = g.c2y[jj], d2y = g.d2y[jj];
                    const T a2z = g.a2z[c], b2z = g.b2z[c], c2z = g.c2z[c], d2z = g.d2z[c];
                    auto L2 = [&](int f) {
                        return d1fc(X(f, 0), X(f, 1), X(f, 2), X(f, 3), X(f, 4), a2x, b2x, c2x, d2x) +
                               d1fc(Y(f, 0), Y(f, 1), Y(f, 2), Y(f, 3), Y(f, 4), a2y, b2y, c2y, d2y) +
                               d1fc(Zz(f, 0), Zz(f, 1), Zz(f, 2), Zz(f, 3), Zz(f, 4), a2z, b2z, c2z, d2z);
                    };
                    out[0] = out[0] + g.drho * (L2(8) + T(g.d2rho0[c]));
                    out[7] = out[7] + g.dp * (L2(4) + T(g.d2p0[c]));
                }
                const long base = (long)i + (long)jj * g.sy;
#pragma unroll
                for (int m = 0; m < NF; ++m) xdif.f[m][cidx] = out[m];
                if (c == 2 || c == mz - 3) {
                    const int kh = c == 2 ? 1 : mz - 2, kz = c == 2 ? 0 : mz - 1;
#pragma unroll
                    for (int m = 0; m < NF; ++m) {
                        xdif.f[m][base + (long)kh * g.sz] = T(0.5) * out[m];
                        xdif.f[m][base + (long)kz * g.sz] = T(0);
                    }
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------------------
// cp.async (sm_80+ asynchronous global->shared copies, kept on sm_100a)
__device__ __forceinline__ void cp_async_elem(float* dst, const float* src) {
    unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src));
}
__device__ __forceinline__ void cp_async_elem(double* dst, const double* src) {
    unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// ---------------------------------------------------------------------------------------
// 16-byte cp.async (one row chunk of 4 floats or 2 doubles)
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src));
}

// radial coefficient, fast FP32 form: 1/32 + (3/32) / (1 + exp(-2u)), u = (r-3)/3, which is
// 1/32 + (3/64)(1 + tanh u) by 1 + tanh u = 2/(1 + exp(-2u)); FP64 keeps tanh
__device__ __forceinline__ float radial_coef_fast(float r2) {
    const float r = sqrtf(r2);
    return 0.03125f + __fdividef(0.09375f, 1.0f + __expf((6.0f - 2.0f * r) * (1.0f / 3.0f)));
}
__device__ __forceinline__ double radial_coef_fast(double r2) { return radial_coef(sqrt(r2)); }

// ---------------------------------------------------------------------------------------
// One smoothing pass (avrg / avrgE / avrgc / avrgh, each followed by its bndry*), z-marching.
// CTA: TX x TYH threads, tile TX x (TYH*RY) columns (each thread RY rows).  Each plane of the
// tile plus its 1-node x/y halo (no corners: the 7-point stencil has none) streams into an
// NS = D + 4 stage shared-memory ring with cp.async, D planes ahead of the plane computed
// (16-byte copies for the tile rows, which start 16-byte aligned in the ring, 4/8-byte
// copies for the two halo columns).  The stage being refilled is never one of the three
// being read, so one barrier per plane suffices.  KINDS: 2 bits per field, 0 radial
// coefficient, 1 constant 1/8, 2 x-profile (B in avrg/avrgtt).  Needs mx % TX == 0.
// MODE 0 writes the smoothed fields.  MODES 1 and 2 are the two passes of avrgtt on a
// compensated FP32 state (x, comp): MODE 1 reads x in fields 0..NF/2-1 and comp in the rest
// and writes the first pass's increment d of x - comp; MODE 2 reads d and hands the two-pass
// increment to a Kahan epilogue (EpiKF).
__host__ __device__ constexpr bool any_kind0(unsigned kinds, int nf) {
    for (int f = 0; f < nf; ++f)
        if (((kinds >> (2 * f)) & 3u) == 0u) return true;
    return false;
}

template <class T, int NF, int TX, int TYH, int RY, int D>
struct ZP {
    static constexpr int TY = TYH * RY;
    static constexpr int OFF = 16 / sizeof(T);        // interior column offset in a ring row
    static constexpr int RS = TX + 2 * OFF;           // ring row stride
    static constexpr int NR = TY + 2;                 // rows: y0-1 .. y0+TY
    static constexpr int SP = RS * NR;                // one field-plane
    static constexpr int NS = D + 4;                  // ring stages (power of two for D = 4)
    static constexpr int CH = TX * (int)sizeof(T) / 16;   // 16-byte chunks per row
    static constexpr size_t smem() { return sizeof(T) * (size_t)NS * NF * SP; }
};

template <class T, int NF, unsigned KINDS, int TX, int TYH, int RY, int D, class Epi, int MODE = 0>
__global__ void __launch_bounds__(TX* TYH) k_zpass(Geo<T> g, SrcFields<T, NF> src, Epi epi, int chunk) {
    using Z = ZP<T, NF, TX, TYH, RY, D>;
    constexpr int RS = Z::RS, SP = Z::SP, NS = Z::NS, OFF = Z::OFF, CH = Z::CH, TY = Z::TY;
    constexpr int NT = TX * TYH;
    constexpr int NO = MODE == 1 ? NF / 2 : NF;       // output fields (MODE 1: x then comp in)
    static_assert(MODE != 1 || NF % 2 == 0, "MODE 1 reads field pairs");
    constexpr int NVEC = Z::NR * CH;                  // vector copies per field-plane
    constexpr int NHAL = 2 * TY;                      // scalar halo-column copies
    static_assert((NS & (NS - 1)) == 0, "ring stages must be a power of two");
    extern __shared__ __align__(16) unsigned char zp_smem_raw[];
    T* ring = reinterpret_cast<T*>(zp_smem_raw);      // [NS][NF][SP]
    const int tid = threadIdx.x;
    const int tx = tid % TX, tyh = tid / TX;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const int mz = g.mz;
    const int k0 = blockIdx.z * chunk;
    const int k1 = min(k0 + chunk, mz);
    const int cA = max(k0, 2), cB = min(k1 - 1, mz - 3);
    if (cA > cB) return;
    // this thread's copy slots (the same for every field and plane)
    constexpr int NSL = (NVEC + NHAL + NT - 1) / NT;
    long gsrc[NSL];
    int sdst[NSL];
#pragma unroll
    for (int q = 0; q < NSL; ++q) {
        const int sl = tid + q * NT;
        gsrc[q] = -1;
        sdst[q] = 0;
        if (sl < NVEC) {
            const int r = sl / CH, ch = sl % CH;
            gsrc[q] = (long)(x0 + ch * (16 / (int)sizeof(T))) + (long)pmod(y0 - 1 + r, g.my) * g.sy;
            sdst[q] = r * RS + OFF + ch * (16 / (int)sizeof(T));
        } else if (sl < NVEC + NHAL) {
            const int h = sl - NVEC, r = h % TY + 1, side = h / TY;
            const int xx = side ? pmod(x0 + TX, g.mx) : pmod(x0 - 1, g.mx);
            gsrc[q] = (long)xx + (long)pmod(y0 - 1 + r, g.my) * g.sy;
            sdst[q] = r * RS + (side ? OFF + TX : OFF - 1);
        }
    }
    const int phi = cB + 1;
    auto issue = [&](int p) {
        if (p <= phi) {
#pragma unroll
            for (int q = 0; q < NSL; ++q) {
                const int sl = tid + q * NT;
                if (sl < NVEC + NHAL) {
                    T* st = ring + (long)(p & (NS - 1)) * NF * SP + sdst[q];
                    const long zo = gsrc[q] + (long)p * g.sz;
#pragma unroll
                    for (int f = 0; f < NF; ++f) {
                        if (sl < NVEC) cp_async16(st + f * SP, src.f[f] + zo);
                        else cp_async_elem(st + f * SP, src.f[f] + zo);
                    }
                }
            }
        }
        cp_async_commit();
    };
#pragma unroll
    for (int p = 0; p < D + 2; ++p) issue(cA - 1 + p);   // planes cA-1 .. cA+D
    const int gi = x0 + tx;
    const T wpx = g.wpx[gi], wmx = g.wmx[gi], cbx = g.cbx[gi];
    const T xx2 = g.xc[gi] * g.xc[gi];
    int gj[RY];
    T wpy[RY], wmy[RY], rr2[RY];
#pragma unroll
    for (int u = 0; u < RY; ++u) {
        gj[u] = y0 + tyh + u * TYH;
        const int jj = gj[u] < g.my ? gj[u] : g.my - 1;
        wpy[u] = g.wpy[jj]; wmy[u] = g.wmy[jj];
        rr2[u] = xx2 + g.yc[jj] * g.yc[jj];
    }
    // per-plane operands, loaded one plane ahead
    T nwpz = g.wpz[cA], nwmz = g.wmz[cA], nzc = g.zc[cA];
    typename Epi::Pre npre[RY];
#pragma unroll
    for (int u = 0; u < RY; ++u)
        if (gj[u] < g.my) epi.pre((long)gi + (long)gj[u] * g.sy + (long)cA * g.sz, npre[u]);
    // own column: planes c-1 and c in registers (z queue); plane c+1 read from the ring
    T qm[RY][NF], q0[RY][NF];
    bool primed = false;
    for (int c = cA; c <= cB; ++c) {
        issue(c + 1 + D);
        const T wpz = nwpz, wmz = nwmz;
        const T zz2 = nzc * nzc;
        typename Epi::Pre cpre[RY];
#pragma unroll
        for (int u = 0; u < RY; ++u) cpre[u] = npre[u];
        if (c < cB) {
            nwpz = g.wpz[c + 1]; nwmz = g.wmz[c + 1]; nzc = g.zc[c + 1];
#pragma unroll
            for (int u = 0; u < RY; ++u)
                if (gj[u] < g.my) epi.pre((long)gi + (long)gj[u] * g.sy + (long)(c + 1) * g.sz, npre[u]);
        }
        cp_async_wait<D>();
        __syncthreads();
        const T* pc = ring + (long)(c & (NS - 1)) * NF * SP;
        const T* pp = ring + (long)((c + 1) & (NS - 1)) * NF * SP;
        if (!primed) {
            const T* pm = ring + (long)((c - 1) & (NS - 1)) * NF * SP;
#pragma unroll
            for (int u = 0; u < RY; ++u) {
                const int me = (tyh + u * TYH + 1) * RS + OFF + tx;
#pragma unroll
                for (int f = 0; f < NF; ++f) { qm[u][f] = pm[f * SP + me]; q0[u][f] = pc[f * SP + me]; }
            }
            primed = true;
        }
#pragma unroll
        for (int u = 0; u < RY; ++u) {
            const int me = (tyh + u * TYH + 1) * RS + OFF + tx;
            T qp[NF];
#pragma unroll
            for (int f = 0; f < NF; ++f) qp[f] = pp[f * SP + me];
            if (gj[u] < g.my) {
                T cr = T(0);
                if (any_kind0(KINDS, NO)) cr = radial_coef_fast(rr2[u] + zz2);
                const long col = (long)gi + (long)gj[u] * g.sy;
                const bool wall = c == 2 || c == mz - 3;
                const int kh = c == 2 ? 1 : mz - 2, kz = c == 2 ? 0 : mz - 1;
                T val[NO];
                if constexpr (MODE == 1) {
                    // increment of the first filter pass on x - comp: differences of x and of
                    // comp taken apart, then combined, so comp's bits are not rounded away
#pragma unroll
                    for (int f = 0; f < NO; ++f) {
                        const T* a = pc + f * SP;
                        const T* b = pc + (f + NO) * SP;
                        const T x0 = q0[u][f], k0 = q0[u][f + NO];
                        const T txp = (a[me + 1] - x0) - (b[me + 1] - k0), txm = (x0 - a[me - 1]) - (k0 - b[me - 1]);
                        const T typ = (a[me + RS] - x0) - (b[me + RS] - k0), tym = (x0 - a[me - RS]) - (k0 - b[me - RS]);
                        const T tzp = (qp[f] - x0) - (qp[f + NO] - k0), tzm = (x0 - qm[u][f]) - (k0 - qm[u][f + NO]);
                        const unsigned kind = (KINDS >> (2 * f)) & 3u;
                        const T coef = kind == 0u ? cr : (kind == 1u ? T(0.125) : cbx);
                        val[f] = coef * (txp * wpx - txm * wmx + typ * wpy[u] - tym * wmy[u] + tzp * wpz - tzm * wmz);
                    }
                    epi.store(g, col + (long)c * g.sz, val, cpre[u]);
                    if (wall) {
                        // wall rows of the pass result: row kh = half of row c, row kz = 0, as
                        // increments of x - comp
                        T hv[NO], zv[NO];
#pragma unroll
                        for (int f = 0; f < NO; ++f) {
                            const T xw = c == 2 ? qm[u][f] : qp[f];
                            const T kw = c == 2 ? qm[u][f + NO] : qp[f + NO];
                            hv[f] = ((T(0.5) * q0[u][f] - xw) - (T(0.5) * q0[u][f + NO] - kw)) + T(0.5) * val[f];
                            const long iz = col + (long)kz * g.sz;
                            zv[f] = src.f[f + NO][iz] - src.f[f][iz];
                        }
                        epi.store(g, col + (long)kh * g.sz, hv);
                        epi.store(g, col + (long)kz * g.sz, zv);
                    }
                } else {
#pragma unroll
                    for (int f = 0; f < NF; ++f) {
                        const T* a = pc + f * SP;
                        const T v0 = q0[u][f];
                        const T tx_ = (a[me + 1] - v0) * wpx - (v0 - a[me - 1]) * wmx;
                        const T ty_ = (a[me + RS] - v0) * wpy[u] - (v0 - a[me - RS]) * wmy[u];
                        const T tz_ = (qp[f] - v0) * wpz - (v0 - qm[u][f]) * wmz;
                        const unsigned kind = (KINDS >> (2 * f)) & 3u;
                        const T coef = kind == 0u ? cr : (kind == 1u ? T(0.125) : cbx);
                        // MODE 2: increment of two passes from the first pass's increment d,
                        // S(S(z)) - z = 2 d + coef L(d)
                        val[f] = (MODE == 2 ? T(2) * v0 : v0) + coef * (tx_ + ty_ + tz_);
                    }
                    if constexpr (MODE == 2) {
                        epi.store_rows(col + (long)c * g.sz, wall, col + (long)kh * g.sz, col + (long)kz * g.sz, val, cpre[u]);
                    } else {
                        epi.store(g, col + (long)c * g.sz, val, cpre[u]);
                        if (wall) {
                            T hv[NF], zv[NF];
#pragma unroll
                            for (int f = 0; f < NF; ++f) { hv[f] = T(0.5) * val[f]; zv[f] = T(0); }
                            epi.store(g, col + (long)kh * g.sz, hv);
                            epi.store(g, col + (long)kz * g.sz, zv);
                        }
                    }
                }
            }
#pragma unroll
            for (int f = 0; f < NF; ++f) { qm[u][f] = q0[u][f]; q0[u][f] = qp[f]; }
        }
    }
    cp_async_wait<0>();
}

}  // namespace dasha

namespace dasha {

// ---------------------------------------------------------------------------------------
// Radius-2 z-marching stencil framework (the RHS of right, t3dsdsc.f:1334-1566).
// CTA TX x TYH threads, one output column each.  NF source fields stream through an
// 8-stage shared-memory ring (tile + 2-node x/y halo, no corners) with cp.async, D = 3
// planes ahead; the op reads planes c-2..c+2 of the ring.  With Op::RINV, field 0 is
// rho - rho0 and a parallel ring holds 1/rho, filled in place by the thread whose copy
// landed each node.
template <class T, int NF, int TX, int TYH>
struct ZS2 {
    static constexpr int OFF = 16 / sizeof(T);
    static constexpr int RS = TX + 2 * OFF;
    static constexpr int NR = TYH + 4;
    static constexpr int SP = RS * NR;
    // D = 2: the stage refilled at plane c (plane c+4) is plane c-4's, which no thread can
    // still be reading (a thread one plane behind reads c-3..c+1)
    static constexpr int NS = 8, D = 2;
    static constexpr int CH = TX * (int)sizeof(T) / 16;
    static constexpr size_t smem(bool rinv) { return sizeof(T) * (size_t)NS * (NF + (rinv ? 1 : 0)) * SP; }
};

template <class T, int NF, int TX, int TYH>
struct ZView {
    using Z = ZS2<T, NF, TX, TYH>;
    const T* st[5];     // stages of planes c-2..c+2
    const T* ri[5];     // 1/rho stages (when present)
    int me;
    // field f at offset s-2 along x, y or z
    __device__ __forceinline__ T X(int f, int s) const { return st[2][f * Z::SP + me + (s - 2)]; }
    __device__ __forceinline__ T Y(int f, int s) const { return st[2][f * Z::SP + me + (s - 2) * Z::RS]; }
    __device__ __forceinline__ T Zz(int f, int s) const { return st[s][f * Z::SP + me]; }
    __device__ __forceinline__ T RX(int s) const { return ri[2][me + (s - 2)]; }
    __device__ __forceinline__ T RY(int s) const { return ri[2][me + (s - 2) * Z::RS]; }
    __device__ __forceinline__ T RZ(int s) const { return ri[s][me]; }
};

template <class T, int NF, int TX, int TYH, int MINB, class Op>
__global__ void __launch_bounds__(TX* TYH, MINB) k_zst2(Geo<T> g, SrcFields<T, NF> src, Op op, int chunk) {
    using Z = ZS2<T, NF, TX, TYH>;
    constexpr int RS = Z::RS, SP = Z::SP, NS = Z::NS, OFF = Z::OFF, CH = Z::CH, D = Z::D;
    constexpr int NT = TX * TYH;
    constexpr int NVEC = Z::NR * CH;
    constexpr int NHAL = 4 * TYH;
    constexpr int NSL = (NVEC + NHAL + NT - 1) / NT;
    constexpr int VE = 16 / (int)sizeof(T);
    constexpr bool RINV = Op::RINV;
    extern __shared__ __align__(16) unsigned char zs2_smem_raw[];
    T* ring = reinterpret_cast<T*>(zs2_smem_raw);        // [NS][NF][SP]
    T* rring = ring + (long)NS * NF * SP;                // [NS][SP] (RINV)
    const int tid = threadIdx.x;
    const int tx = tid % TX, ty = tid / TX;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TYH;
    const int mz = g.mz;
    const int k0 = blockIdx.z * chunk;
    const int k1 = min(k0 + chunk, mz);
    const int cA = max(k0, 2), cB = min(k1 - 1, mz - 3);
    if (cA > cB) return;
    long gsrc[NSL];
    int sdst[NSL];
#pragma unroll
    for (int q = 0; q < NSL; ++q) {
        const int sl = tid + q * NT;
        gsrc[q] = -1;
        sdst[q] = 0;
        if (sl < NVEC) {
            const int r = sl / CH, ch = sl % CH;
            gsrc[q] = (long)(x0 + ch * VE) + (long)pmod(y0 - 2 + r, g.my) * g.sy;
            sdst[q] = r * RS + OFF + ch * VE;
        } else if (sl < NVEC + NHAL) {
            const int h = sl - NVEC, r = h % TYH + 2, side = h / TYH;   // side 0..3: x0-2, x0-1, x0+TX, x0+TX+1
            const int dxo = side < 2 ? side - 2 : TX + side - 2;
            gsrc[q] = (long)pmod(x0 + dxo, g.mx) + (long)pmod(y0 - 2 + r, g.my) * g.sy;
            sdst[q] = r * RS + OFF + dxo;
        }
    }
    const int phi = cB + 2;
    auto issue = [&](int p) {
        if (p <= phi) {
#pragma unroll
            for (int q = 0; q < NSL; ++q) {
                const int sl = tid + q * NT;
                if (sl < NVEC + NHAL) {
                    T* st = ring + (long)(p & (NS - 1)) * NF * SP + sdst[q];
                    const long zo = gsrc[q] + (long)p * g.sz;
#pragma unroll
                    for (int f = 0; f < NF; ++f) {
                        if (sl < NVEC) cp_async16(st + f * SP, src.f[f] + zo);
                        else cp_async_elem(st + f * SP, src.f[f] + zo);
                    }
                }
            }
        }
        cp_async_commit();
    };
    // 1/rho of the nodes this thread copied in plane p (its own copies have landed)
    auto make_rinv = [&](int p) {
        if (!RINV) return;
        const T r0 = T(g.rho0[p]);
        const T* dr = ring + (long)(p & (NS - 1)) * NF * SP;
        T* ri = rring + (long)(p & (NS - 1)) * SP;
#pragma unroll
        for (int q = 0; q < NSL; ++q) {
            const int sl = tid + q * NT;
            if (sl < NVEC) {
#pragma unroll
                for (int e = 0; e < VE; ++e) ri[sdst[q] + e] = T(1) / (r0 + dr[sdst[q] + e]);
            } else if (sl < NVEC + NHAL) {
                ri[sdst[q]] = T(1) / (r0 + dr[sdst[q]]);
            }
        }
    };
#pragma unroll
    for (int p = 0; p < D + 4; ++p) issue(cA - 2 + p);      // planes cA-2 .. cA+1+D
    const int gi = x0 + tx, gj = y0 + ty;
    const bool out_ok = gj < g.my;
    const int jj = out_ok ? gj : g.my - 1;
    typename Op::Col col;
    op.column(g, gi, jj, col);
    typename Op::Pre npre;
    op.pre(g, gi, jj, cA, npre);
    ZView<T, NF, TX, TYH> v;
    v.me = (ty + 2) * RS + OFF + tx;
    for (int c = cA; c <= cB; ++c) {
        issue(c + 2 + D);
        const typename Op::Pre cpre = npre;
        if (c < cB) op.pre(g, gi, jj, c + 1, npre);
        cp_async_wait<D>();
        if (RINV) {
            if (c == cA)
                for (int p = c - 2; p <= c + 2; ++p) make_rinv(p);
            else
                make_rinv(c + 2);
        }
        __syncthreads();
#pragma unroll
        for (int s = 0; s < 5; ++s) {
            v.st[s] = ring + (long)((c - 2 + s) & (NS - 1)) * NF * SP;
            v.ri[s] = rring + (long)((c - 2 + s) & (NS - 1)) * SP;
        }
        if (out_ok) op.compute(g, v, gi, jj, c, col, cpre);
    }
    cp_async_wait<0>();
}

// SIGN * curl of the 3 ring fields, wall rows applied: SIGN = +1 is J1 = curl(B - B0)
// (current t3dsdsc.f:2476-2491 with bndryc), SIGN = -1 is dB/dt = -curl E (t3dsdsc.f:1435-1452)
template <class T, int SIGN>
struct OpCurl {
    static constexpr bool RINV = false;
    T* out[3];
    struct Col { T ax, bx, cx, dx, ay, by, cy, dy; };
    struct Pre { T az, bz, cz, dz; };
    __device__ __forceinline__ void column(const Geo<T>& g, int i, int j, Col& c) const {
        c.ax = g.a1x[i]; c.bx = g.b1x[i]; c.cx = g.c1x[i]; c.dx = g.d1x[i];
        c.ay = g.a1y[j]; c.by = g.b1y[j]; c.cy = g.c1y[j]; c.dy = g.d1y[j];
    }
    __device__ __forceinline__ void pre(const Geo<T>& g, int, int, int c, Pre& p) const {
        p.az = g.a1z[c]; p.bz = g.b1z[c]; p.cz = g.c1z[c]; p.dz = g.d1z[c];
    }
    template <class V>
    __device__ __forceinline__ void compute(const Geo<T>& g, const V& v, int i, int j, int c, const Col& k,
                                            const Pre& p) const {
        auto DX = [&](int f) { return d1fc(v.X(f, 0), v.X(f, 1), v.X(f, 2), v.X(f, 3), v.X(f, 4), k.ax, k.bx, k.cx, k.dx); };
        auto DY = [&](int f) { return d1fc(v.Y(f, 0), v.Y(f, 1), v.Y(f, 2), v.Y(f, 3), v.Y(f, 4), k.ay, k.by, k.cy, k.dy); };
        auto DZ = [&](int f) { return d1fc(v.Zz(f, 0), v.Zz(f, 1), v.Zz(f, 2), v.Zz(f, 3), v.Zz(f, 4), p.az, p.bz, p.cz, p.dz); };
        T o[3];
        if (SIGN > 0) {
            o[0] = DY(2) - DZ(1);
            o[1] = DZ(0) - DX(2);
            o[2] = DX(1) - DY(0);
        } else {
            o[0] = -DY(2) + DZ(1);
            o[1] = -DZ(0) + DX(2);
            o[2] = -DX(1) + DY(0);
        }
        const long base = (long)i + (long)j * g.sy;
#pragma unroll
        for (int m = 0; m < 3; ++m) out[m][base + (long)c * g.sz] = o[m];
        if (c == 2 || c == g.mz - 3) {
            const int kh = c == 2 ? 1 : g.mz - 2, kz = c == 2 ? 0 : g.mz - 1;
#pragma unroll
            for (int m = 0; m < 3; ++m) {
                out[m][base + (long)kh * g.sz] = T(0.5) * o[m];
                out[m][base + (long)kz * g.sz] = T(0);
            }
        }
    }
};

// Hall term xdh = di (J x B - grad p) / rho with the wall rows (t3dsdsc.f:1404-1423, bndryh);
// ring field dp, the rest pointwise
template <class T>
struct OpHall {
    static constexpr bool RINV = false;
    T* out[3];
    const T *r, *b1, *b2, *b3, *j1, *j2, *j3;
    struct Col { T ax, bx, cx, dx, ay, by, cy, dy; };
    struct Pre { T az, bz, cz, dz, r, b1, b2, b3, j1, j2, j3, dzp0; };
    __device__ __forceinline__ void column(const Geo<T>& g, int i, int j, Col& c) const {
        c.ax = g.a1x[i]; c.bx = g.b1x[i]; c.cx = g.c1x[i]; c.dx = g.d1x[i];
        c.ay = g.a1y[j]; c.by = g.b1y[j]; c.cy = g.c1y[j]; c.dy = g.d1y[j];
    }
    __device__ __forceinline__ void pre(const Geo<T>& g, int i, int j, int c, Pre& p) const {
        const long ci = (long)i + (long)j * g.sy + (long)c * g.sz;
        p.az = g.a1z[c]; p.bz = g.b1z[c]; p.cz = g.c1z[c]; p.dz = g.d1z[c];
        p.r = T(g.rho0[c]) + r[ci];
        p.b1 = T(g.bx0[c]) + b1[ci]; p.b2 = T(g.by0[c]) + b2[ci]; p.b3 = T(g.bz0[c]) + b3[ci];
        p.j1 = j1[ci]; p.j2 = j2[ci]; p.j3 = j3[ci];
        p.dzp0 = T(g.dzp0[c]);
    }
    template <class V>
    __device__ __forceinline__ void compute(const Geo<T>& g, const V& v, int i, int j, int c, const Col& k,
                                            const Pre& p) const {
        const T px = d1fc(v.X(0, 0), v.X(0, 1), v.X(0, 2), v.X(0, 3), v.X(0, 4), k.ax, k.bx, k.cx, k.dx);
        const T py = d1fc(v.Y(0, 0), v.Y(0, 1), v.Y(0, 2), v.Y(0, 3), v.Y(0, 4), k.ay, k.by, k.cy, k.dy);
        const T pz = d1fc(v.Zz(0, 0), v.Zz(0, 1), v.Zz(0, 2), v.Zz(0, 3), v.Zz(0, 4), p.az, p.bz, p.cz, p.dz) + p.dzp0;
        T o[3];
        o[0] = g.di * (p.j2 * p.b3 - p.j3 * p.b2 - px) / p.r;
        o[1] = g.di * (p.j3 * p.b1 - p.j1 * p.b3 - py) / p.r;
        o[2] = g.di * (p.j1 * p.b2 - p.j2 * p.b1 - pz) / p.r;
        const long base = (long)i + (long)j * g.sy;
#pragma unroll
        for (int m = 0; m < 3; ++m) out[m][base + (long)c * g.sz] = o[m];
        if (c == 2 || c == g.mz - 3) {
            const int kh = c == 2 ? 1 : g.mz - 2, kz = c == 2 ? 0 : g.mz - 1;
#pragma unroll
            for (int m = 0; m < 3; ++m) {
                out[m][base + (long)kh * g.sz] = T(0.5) * o[m];
                out[m][base + (long)kz * g.sz] = T(0);
            }
        }
    }
};

// continuity, momentum (flux t3dsdsc.f:2304-2347, J x B - xresd t3dsdsc.f:1355-1360) and
// pressure (t3dsdsc.f:1550-1566), with the optional viscous / diffusive terms
// (t3dsdsc.f:1585-1663); ring fields drho m1 m2 m3 dp (+ 1/rho)
template <class T>
struct OpHydro {
    static constexpr bool RINV = true;
    T* out[5];                  // xdif 0 1 2 3 7
    const T *j1, *j2, *j3, *b1, *b2, *b3;
    struct Col { T ax, bx, cx, dx, ay, by, cy, dy; };
    struct Pre { T az, bz, cz, dz, j1, j2, j3, b1, b2, b3, rsx, rsy, rsz, dzp0, p0; };
    __device__ __forceinline__ void column(const Geo<T>& g, int i, int j, Col& c) const {
        c.ax = g.a1x[i]; c.bx = g.b1x[i]; c.cx = g.c1x[i]; c.dx = g.d1x[i];
        c.ay = g.a1y[j]; c.by = g.b1y[j]; c.cy = g.c1y[j]; c.dy = g.d1y[j];
    }
    __device__ __forceinline__ void pre(const Geo<T>& g, int i, int j, int c, Pre& p) const {
        const long ci = (long)i + (long)j * g.sy + (long)c * g.sz;
        p.az = g.a1z[c]; p.bz = g.b1z[c]; p.cz = g.c1z[c]; p.dz = g.d1z[c];
        p.j1 = j1[ci]; p.j2 = j2[ci]; p.j3 = j3[ci];
        p.b1 = T(g.bx0[c]) + b1[ci]; p.b2 = T(g.by0[c]) + b2[ci]; p.b3 = T(g.bz0[c]) + b3[ci];
        p.rsx = T(g.rsx[c]); p.rsy = T(g.rsy[c]); p.rsz = T(g.rsz[c]); p.dzp0 = T(g.dzp0[c]); p.p0 = T(g.p0[c]);
    }
    template <class V>
    __device__ __forceinline__ void compute(const Geo<T>& g, const V& v, int i, int j, int c, const Col& k,
                                            const Pre& p) const {
        auto DX = [&](auto fn) { return d1fc(fn(0), fn(1), fn(2), fn(3), fn(4), k.ax, k.bx, k.cx, k.dx); };
        auto DY = [&](auto fn) { return d1fc(fn(0), fn(1), fn(2), fn(3), fn(4), k.ay, k.by, k.cy, k.dy); };
        auto DZ = [&](auto fn) { return d1fc(fn(0), fn(1), fn(2), fn(3), fn(4), p.az, p.bz, p.cz, p.dz); };
        T o[5];
        // fields: 0 drho, 1 m1, 2 m2, 3 m3, 4 dp
        o[0] = -DX([&](int s) { return v.X(1, s); }) - DY([&](int s) { return v.Y(2, s); }) -
               DZ([&](int s) { return v.Zz(3, s); });
        o[1] = -DX([&](int s) { return v.X(1, s) * v.X(1, s) * v.RX(s) + v.X(4, s); }) -
               DY([&](int s) { return v.Y(1, s) * v.Y(2, s) * v.RY(s); }) -
               DZ([&](int s) { return v.Zz(1, s) * v.Zz(3, s) * v.RZ(s); });
        o[2] = -DX([&](int s) { return v.X(1, s) * v.X(2, s) * v.RX(s); }) -
               DY([&](int s) { return v.Y(2, s) * v.Y(2, s) * v.RY(s) + v.Y(4, s); }) -
               DZ([&](int s) { return v.Zz(2, s) * v.Zz(3, s) * v.RZ(s); });
        o[3] = -DX([&](int s) { return v.X(1, s) * v.X(3, s) * v.RX(s); }) -
               DY([&](int s) { return v.Y(2, s) * v.Y(3, s) * v.RY(s); }) -
               DZ([&](int s) { return v.Zz(3, s) * v.Zz(3, s) * v.RZ(s) + v.Zz(4, s); });
        o[1] = o[1] - p.rsx + p.j2 * p.b3 - p.j3 * p.b2;
        o[2] = o[2] - p.rsy + p.j3 * p.b1 - p.j1 * p.b3;
        o[3] = o[3] - p.rsz + p.j1 * p.b2 - p.j2 * p.b1;
        const T ri = v.RX(2);
        const T v1 = v.X(1, 2) * ri, v2 = v.X(2, 2) * ri, v3 = v.X(3, 2) * ri;
        const T px = DX([&](int s) { return v.X(4, s); });
        const T py = DY([&](int s) { return v.Y(4, s); });
        const T pz = DZ([&](int s) { return v.Zz(4, s); }) + p.dzp0;
        const T divv = -DX([&](int s) { return v.X(1, s) * v.RX(s); }) - DY([&](int s) { return v.Y(2, s) * v.RY(s); }) -
                       DZ([&](int s) { return v.Zz(3, s) * v.RZ(s); });
        const T pc = p.p0 + v.X(4, 2);
        o[4] = -px * v1 - py * v2 - pz * v3 + divv * g.gamma * pc +
               (g.gamma - T(1)) * g.eta * (p.j1 * p.j1 + p.j2 * p.j2 + p.j3 * p.j3);
        if (g.viscos) {
            const T a2x = g.a2x[i], b2x = g.b2x[i], c2x = g.c2x[i], d2x = g.d2x[i];
            const T a2y = g.a2y[j], b2y = g.b2y[j], c2y = g.c2y[j], d2y = g.d2y[j];
            const T a2z = g.a2z[c], b2z = g.b2z[c], c2z = g.c2z[c], d2z = g.d2z[c];
            auto L = [&](int f) {
                return d1fc(v.X(f, 0) * v.RX(0), v.X(f, 1) * v.RX(1), v.X(f, 2) * v.RX(2), v.X(f, 3) * v.RX(3),
                            v.X(f, 4) * v.RX(4), a2x, b2x, c2x, d2x) +
                       d1fc(v.Y(f, 0) * v.RY(0), v.Y(f, 1) * v.RY(1), v.Y(f, 2) * v.RY(2), v.Y(f, 3) * v.RY(3),
                            v.Y(f, 4) * v.RY(4), a2y, b2y, c2y, d2y) +
                       d1fc(v.Zz(f, 0) * v.RZ(0), v.Zz(f, 1) * v.RZ(1), v.Zz(f, 2) * v.RZ(2), v.Zz(f, 3) * v.RZ(3),
                            v.Zz(f, 4) * v.RZ(4), a2z, b2z, c2z, d2z);
            };
            const T af = L(1), ag = L(2), ah = L(3);
            o[1] = o[1] + g.mu * af;
            o[2] = o[2] + g.mu * ag;
            o[3] = o[3] + g.mu * ah;
            o[4] = o[4] + g.mu * (v1 * af + v2 * ag + v3 * ah);
        }
        if (g.diffu) {
            const T a2x = g.a2x[i], b2x = g.b2x[i], c2x = g.c2x[i], d2x = g.d2x[i];
            const T a2y = g.a2y[j], b2y = g.b2y[j], c2y = g.c2y[j], d2y = g.d2y[j];
            const T a2z = g.a2z[c], b2z = g.b2z[c], c2z = g.c2z[c], d2z = g.d2z[c];
            auto L2 = [&](int f) {
                return d1fc(v.X(f, 0), v.X(f, 1), v.X(f, 2), v.X(f, 3), v.X(f, 4), a2x, b2x, c2x, d2x) +
                       d1fc(v.Y(f, 0), v.Y(f, 1), v.Y(f, 2), v.Y(f, 3), v.Y(f, 4), a2y, b2y, c2y, d2y) +
                       d1fc(v.Zz(f, 0), v.Zz(f, 1), v.Zz(f, 2), v.Zz(f, 3), v.Zz(f, 4), a2z, b2z, c2z, d2z);
            };
            o[0] = o[0] + g.drho * (L2(0) + T(g.d2rho0[c]));
            o[4] = o[4] + g.dp * (L2(4) + T(g.d2p0[c]));
        }
        const long base = (long)i + (long)j * g.sy;
#pragma unroll
        for (int m = 0; m < 5; ++m) out[m][base + (long)c * g.sz] = o[m];
        if (c == 2 || c == g.mz - 3) {
            const int kh = c == 2 ? 1 : g.mz - 2, kz = c == 2 ? 0 : g.mz - 1;
#pragma unroll
            for (int m = 0; m < 5; ++m) {
                out[m][base + (long)kh * g.sz] = T(0.5) * o[m];
                out[m][base + (long)kz * g.sz] = T(0);
            }
        }
    }
};

}  // namespace dasha
