// mhd_kernels.cuh -- sm_100a kernels of the RK4 Hall-MHD step (reference: t3dsdsc.f).
//
// Storage: structure-of-arrays, one array per field, node (i,j,k) at i + mx*(j + my*k),
// no ghost nodes.  x and y are periodic (index wrap); z rows 0,1,mz-2,mz-1 are the wall
// rows of the reference (outer row 0, next row one half of its inner neighbour).
// Every field is stored as the perturbation from the FP64 z-profile equilibrium
// (rho0, B0, p0; momentum has no equilibrium part), in type T (double or float).
//
// Each kernel is launched on a 3-D grid: blockIdx.x covers x in chunks of blockDim.x,
// blockIdx.y = j, blockIdx.z = k, so a warp reads consecutive x (coalesced).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace dasha {

constexpr int NF = 8;

template <class T>
struct Geo {
    int mx, my, mz;
    long sy, sz;
    // 4th-order first / second derivative coefficients (t3dsdsc.f:336-504), zero where the
    // reference leaves them undefined (z rows outside 2..mz-3)
    const T *a1x, *b1x, *c1x, *d1x, *a1y, *b1y, *c1y, *d1y, *a1z, *b1z, *c1z, *d1z;
    const T *a2x, *b2x, *c2x, *d2x, *a2y, *b2y, *c2y, *d2y, *a2z, *b2z, *c2z, *d2z;
    // difc weights: difc = (f+ - f0)*wp - (f0 - f-)*wm  (t3dsdsc.f:5618-5619)
    const T *wpx, *wmx, *wpy, *wmy, *wpz, *wmz;
    const T *cbx;    // (1/32)(1 - tanh((x+3)/8)), smoothing coefficient of B (t3dsdsc.f:5636-5642)
    const T *xc, *yc, *zc;   // node coordinates: the radial coefficient 1/32 + 3/32 (1 + tanh((r-3)/3))/2
                             // (t3dsdsc.f:5659-5661) is evaluated per node, not stored
    // equilibrium z-profiles (FP64)
    const double *rho0, *bx0, *by0, *bz0, *p0;
    const double *dzp0;               // Dz p0 (interior rows)
    const double *d2rho0, *d2p0;      // D2z rho0, D2z p0 (interior rows)
    const double *rsx, *rsy, *rsz;    // xresd profiles (interior rows)
    const double *j0x, *j0y, *j0z;    // J0 profiles for j0_mode FULL (null otherwise)
    const double *dzp0r;              // Dz p0 / rho0 (interior rows)
    T eta, di, gamma, mu, drho, dp;
    int hall, viscos, diffu;
    // first plane of setdt's region: 0, except on a z-slab above the lowest one, whose planes 0
    // and 1 are ghost copies of the slab below (halo.h)
    int kcfl0;
};

template <class T>
struct F8 { T* f[NF]; };
template <class T>
struct F3 { T* f[3]; };

__device__ __forceinline__ int wrapi(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

// -DDASHA_BOUNDS (a checking build for tests): the z-marching kernels test every global node
// span they load or store against the field extent n; the first violation of a launch is kept
// in g_bounds_hit as (site + 1) << 48 | index, the access is skipped (no trap, no fault), and the
// C-ABI call that launched it returns DASHA_E_CUDA naming the site and index.  In the normal
// build DASHA_SPAN is `true` and costs nothing.
enum BoundsSite {
    BS_ZPV_LOAD, BS_ZPV_STORE, BS_ZPV_WALL_LOAD, BS_ZPV2_LOAD, BS_ZPV2_STORE, BS_ZCURL_LOAD, BS_ZCURL_STORE,
    BS_ZHYDRO_LOAD, BS_ZHYDRO_NODE_LOAD, BS_ZHYDRO_STORE, BS_ZEH_LOAD, BS_ZEH_NODE_LOAD, BS_ZEH_STORE, BS_COUNT
};
#ifdef DASHA_BOUNDS
static __device__ unsigned long long g_bounds_hit;
__device__ __forceinline__ bool dasha_span(long first, long count, long n, int site) {
    if (first >= 0 && first + count <= n) return true;
    atomicCAS(&g_bounds_hit, 0ull, ((unsigned long long)(site + 1) << 48) | ((unsigned long long)first & 0xFFFFFFFFFFFFull));
    return false;
}
#define DASHA_SPAN(first, count, n, site) dasha_span((long)(first), (long)(count), (long)(n), (int)(site))
#else
#define DASHA_SPAN(first, count, n, site) true
#endif

template <class T>
__device__ __forceinline__ T d1fc(T fm2, T fm, T f0, T fp, T fp2, T a, T b, T c, T d) {
    return a * (fp - f0) + b * (f0 - fm) + c * (fp2 - f0) + d * (f0 - fm2);
}

// d1fc on two FP32 values at once (packed FADD2 / FMUL2 / FFMA2 on sm_100): a (fp - f0), then
// + b (f0 - fm), + c (fp2 - f0), + d (f0 - fm2) by fused multiply-adds.  (Spelling the scalar
// form the same way made the FP64 hydro RHS 25 % slower on B200: one serial chain of DFMAs.)
__device__ __forceinline__ float2 neg2(float2 v) { return make_float2(-v.x, -v.y); }
__device__ __forceinline__ float2 d1fc2(float2 fm2, float2 fm, float2 f0, float2 fp, float2 fp2, float2 a, float2 b,
                                        float2 c, float2 d) {
    float2 t = __fmul2_rn(a, __fadd2_rn(fp, neg2(f0)));
    t = __ffma2_rn(b, __fadd2_rn(f0, neg2(fm)), t);
    t = __ffma2_rn(c, __fadd2_rn(fp2, neg2(f0)), t);
    return __ffma2_rn(d, __fadd2_rn(f0, neg2(fm2)), t);
}
__device__ __forceinline__ float2 bc2(float v) { return make_float2(v, v); }

// 1/v rounded to nearest: the same value as the IEEE division 1/v, without its slow path
__device__ __forceinline__ float recip(float v) { return __frcp_rn(v); }
__device__ __forceinline__ double recip(double v) { return __drcp_rn(v); }

// Stencil helper: neighbour offsets of node (i,j,k) in a periodic-x/y, bounded-z array.
template <class T>
struct Nbr {
    long c;              // centre
    long xm2, xm1, xp1, xp2, ym2, ym1, yp1, yp2;   // absolute indices
    int i, j, k;
    __device__ __forceinline__ Nbr(const Geo<T>& g, int i_, int j_, int k_) : i(i_), j(j_), k(k_) {
        long row = (long)j * g.sy + (long)k * g.sz;
        c = row + i;
        xm2 = row + wrapi(i - 2, g.mx); xm1 = row + wrapi(i - 1, g.mx);
        xp1 = row + wrapi(i + 1, g.mx); xp2 = row + wrapi(i + 2, g.mx);
        long col = (long)i + (long)k * g.sz;
        ym2 = col + (long)wrapi(j - 2, g.my) * g.sy; ym1 = col + (long)wrapi(j - 1, g.my) * g.sy;
        yp1 = col + (long)wrapi(j + 1, g.my) * g.sy; yp2 = col + (long)wrapi(j + 2, g.my) * g.sy;
    }
    __device__ __forceinline__ T Dx(const Geo<T>& g, const T* f) const {
        return d1fc(f[xm2], f[xm1], f[c], f[xp1], f[xp2], g.a1x[i], g.b1x[i], g.c1x[i], g.d1x[i]);
    }
    __device__ __forceinline__ T Dy(const Geo<T>& g, const T* f) const {
        return d1fc(f[ym2], f[ym1], f[c], f[yp1], f[yp2], g.a1y[j], g.b1y[j], g.c1y[j], g.d1y[j]);
    }
    __device__ __forceinline__ T Dz(const Geo<T>& g, const T* f) const {
        return d1fc(f[c - 2 * g.sz], f[c - g.sz], f[c], f[c + g.sz], f[c + 2 * g.sz],
                    g.a1z[k], g.b1z[k], g.c1z[k], g.d1z[k]);
    }
    __device__ __forceinline__ T D2x(const Geo<T>& g, const T* f) const {
        return d1fc(f[xm2], f[xm1], f[c], f[xp1], f[xp2], g.a2x[i], g.b2x[i], g.c2x[i], g.d2x[i]);
    }
    __device__ __forceinline__ T D2y(const Geo<T>& g, const T* f) const {
        return d1fc(f[ym2], f[ym1], f[c], f[yp1], f[yp2], g.a2y[j], g.b2y[j], g.c2y[j], g.d2y[j]);
    }
    __device__ __forceinline__ T D2z(const Geo<T>& g, const T* f) const {
        return d1fc(f[c - 2 * g.sz], f[c - g.sz], f[c], f[c + g.sz], f[c + 2 * g.sz],
                    g.a2z[k], g.b2z[k], g.c2z[k], g.d2z[k]);
    }
    // one Jacobi smoothing stencil: difc_x + difc_y + difc_z (t3dsdsc.f:5643-5648)
    __device__ __forceinline__ T difc3(const Geo<T>& g, const T* f) const {
        T f0 = f[c];
        T tx = (f[xp1] - f0) * g.wpx[i] - (f0 - f[xm1]) * g.wmx[i];
        T ty = (f[yp1] - f0) * g.wpy[j] - (f0 - f[ym1]) * g.wmy[j];
        T tz = (f[c + g.sz] - f0) * g.wpz[k] - (f0 - f[c - g.sz]) * g.wmz[k];
        return tx + ty + tz;
    }
};

// Row rule of the z walls: which interior row a wall row copies from, and the factor.
__device__ __forceinline__ int wall_src(int k, int mz, bool& zero, bool& half) {
    zero = (k == 0 || k == mz - 1);
    half = (k == 1 || k == mz - 2);
    if (k == 1) return 2;
    if (k == mz - 2) return mz - 3;
    return k;
}

// ---------------------------------------------------------------------------------------
// J1 = curl(B - B0) on interior rows + wall rows (current t3dsdsc.f:2468-2491, bndryc).
template <class T>
__global__ void k_curl(Geo<T> g, F3<T> b, F3<T> j) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.mx) return;
    int jj = blockIdx.y, k = blockIdx.z;
    bool zero, half;
    int ks = wall_src(k, g.mz, zero, half);
    long c = (long)i + (long)jj * g.sy + (long)k * g.sz;
    if (zero) { j.f[0][c] = T(0); j.f[1][c] = T(0); j.f[2][c] = T(0); return; }
    Nbr<T> n(g, i, jj, ks);
    T cx = n.Dy(g, b.f[2]) - n.Dz(g, b.f[1]);
    T cy = n.Dz(g, b.f[0]) - n.Dx(g, b.f[2]);
    T cz = n.Dx(g, b.f[1]) - n.Dy(g, b.f[0]);
    if (half) { cx = T(0.5) * cx; cy = T(0.5) * cy; cz = T(0.5) * cz; }
    j.f[0][c] = cx; j.f[1][c] = cy; j.f[2][c] = cz;
}

// ---------------------------------------------------------------------------------------
// NFLD field pointers (the transposed smoothing passes of the adjoint)
template <class T, int NFLD>
struct FS { T* f[NFLD]; };

// ---------------------------------------------------------------------------------------
// E = -v x B + eta*J at every node (t3dsdsc.f:1367-1372).
template <class T>
__global__ void k_efield(Geo<T> g, F8<T> x, F3<T> cur, F3<T> e) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.mx) return;
    int jj = blockIdx.y, k = blockIdx.z;
    long c = (long)i + (long)jj * g.sy + (long)k * g.sz;
    T r = T(g.rho0[k]) + x.f[0][c];
    T m1 = x.f[1][c], m2 = x.f[2][c], m3 = x.f[3][c];
    T b1 = T(g.bx0[k]) + x.f[4][c], b2 = T(g.by0[k]) + x.f[5][c], b3 = T(g.bz0[k]) + x.f[6][c];
    const T ri = T(1) / r;
    e.f[0][c] = (-m2 * b3 + m3 * b2) * ri + g.eta * cur.f[0][c];
    e.f[1][c] = (-m3 * b1 + m1 * b3) * ri + g.eta * cur.f[1][c];
    e.f[2][c] = (-m1 * b2 + m2 * b1) * ri + g.eta * cur.f[2][c];
}

// ---------------------------------------------------------------------------------------
// J0 added to the smoothed J1 (j0_mode FULL).
template <class T>
__global__ void k_add_j0(Geo<T> g, F3<T> cur) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.mx) return;
    int jj = blockIdx.y, k = blockIdx.z;
    long c = (long)i + (long)jj * g.sy + (long)k * g.sz;
    cur.f[0][c] += T(g.j0x[k]);
    cur.f[1][c] += T(g.j0y[k]);
    cur.f[2][c] += T(g.j0z[k]);
}

// ---------------------------------------------------------------------------------------
// FP64 reductions
__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_down_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// CFL in rate form: the reference's per-direction step h / (vp/cfl + visc/(2h)) is the
// inverse of the rate vp * (1/(cfl h)) + visc/(2 h^2), so dt = min(100, 1 / max rate) over
// the region k 0..mz-3, j 0..my-2, i 0..mx-3 (t3dsdsc.f:4709-4736).  Tables per axis:
// ich = 1/(cfl |h|), vv = visc/(2 h^2), ih = 1/|h| (whistler term).  One block per (j,k)
// row; NaN wins so that a corrupted state is reported.
__device__ __forceinline__ double nanmax(double a, double b) { return (a != a || b != b) ? (a != a ? a : b) : fmax(a, b); }

// The CFL rate of node c (totals = equilibrium profile at the node's plane + stored
// perturbation), max over the three directions; shared by k_cfl_rate and the fused tap.
template <class T>
__device__ __forceinline__ double cfl_node_rate(const F8<T>& x, long c, double r0, double bx0, double by0, double bz0,
                                                double p0, double gamma, double whistler, double cx, double vx_,
                                                double hx, double cy, double vy_, double hy, double cz, double vz_,
                                                double hz) {
    double rinv = 1.0 / (r0 + (double)x.f[0][c]);
    double vx = (double)x.f[1][c] * rinv, vy = (double)x.f[2][c] * rinv, vz = (double)x.f[3][c] * rinv;
    double b1 = bx0 + (double)x.f[4][c], b2 = by0 + (double)x.f[5][c], b3 = bz0 + (double)x.f[6][c];
    double bb = b1 * b1 + b2 * b2 + b3 * b3;
    double vf = sqrt(fabs((bb + gamma * (p0 + (double)x.f[7][c])) * rinv));
    double w = whistler != 0.0 ? whistler * sqrt(bb) * rinv : 0.0;
    double rx = (fabs(vx) + vf + w * hx) * cx + vx_;
    double ry = (fabs(vy) + vf + w * hy) * cy + vy_;
    double rz = (fabs(vz) + vf + w * hz) * cz + vz_;
    return nanmax(rx, nanmax(ry, rz));
}

// The fused form of setdt's sweep (survey row f3): the step's last launch, after it stores the
// final B and p of a node (rho and rho v of the node were finished by the launch before it),
// reads the node's 8 fields back and folds its CFL rate into a running maximum; at the end of
// the launch each CTA adds its maximum with one atomicMax on the bits of a double (rates are
// >= 0, so their bit patterns order as unsigned integers, and a NaN pattern lies above every
// finite one: NaN wins as in k_cfl_rate).  The next dasha_setdt then needs no pass over the
// state.  Region and formula as k_cfl_rate.
template <class T>
struct CflTap {
    F8<T> x;
    const double *ich, *vv, *ih;   // per-axis tables, x | y | z concatenated
    const double *rho0, *bx0, *by0, *bz0, *p0;
    double gamma, whistler;
    int mx, my, mz;
    unsigned sy, sz;
    unsigned long long* out;
    __device__ __forceinline__ double rate(long i) const {
        const unsigned n = (unsigned)i, k = n / sz, r = n - k * sz, j = r / sy, ix = r - j * sy;
        if ((int)k > mz - 3 || (int)j > my - 2 || (int)ix > mx - 3) return 0.0;
        const double *iy = ich + mx, *iz = ich + mx + my, *wy = vv + mx, *wz = vv + mx + my;
        const double *hy = ih + mx, *hz = ih + mx + my;
        return cfl_node_rate(x, i, rho0[k], bx0[k], by0[k], bz0[k], p0[k], gamma, whistler, ich[ix], vv[ix], ih[ix],
                             iy[j], wy[j], hy[j], iz[k], wz[k], hz[k]);
    }
};

// An epilogue with the tap: stores through Inner, then takes the rate of each stored node
template <class Inner, class T, int VX>
struct WithCfl : Inner {
    CflTap<T> tap;
    mutable double best;
    using Pre = typename Inner::Pre;
    __device__ __forceinline__ void take(long i) const {
#pragma unroll
        for (int e = 0; e < VX; ++e) best = nanmax(best, tap.rate(i + e));
    }
    template <class V>
    __device__ __forceinline__ void store(long i, const V& v, const Pre& p) const { Inner::store(i, v, p); take(i); }
    template <class V>
    __device__ __forceinline__ void wall(long i, const V& v) const { Inner::wall(i, v); take(i); }
    template <class V>
    __device__ __forceinline__ void store_rows(long i, bool wall, long ih, long iz, const V& v, const Pre& p) const {
        Inner::store_rows(i, wall, ih, iz, v, p);
        take(i);
        if (wall) { take(ih); take(iz); }
    }
    // every thread of the CTA, after its last store
    __device__ __forceinline__ void finish() const {
        __shared__ double sh[32];
        double v = best;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = nanmax(v, __shfl_down_sync(0xffffffffu, v, o));
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        if (lane == 0) sh[wid] = v;
        __syncthreads();
        if (wid == 0) {
            const int nw = (blockDim.x + 31) >> 5;
            v = lane < nw ? sh[lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v = nanmax(v, __shfl_down_sync(0xffffffffu, v, o));
            if (lane == 0 && v != 0.0) atomicMax(tap.out, (unsigned long long)__double_as_longlong(v));
        }
    }
};

template <class E, class = void>
struct has_finish { static constexpr bool value = false; };
template <class E>
struct has_finish<E, decltype((void)&E::finish)> { static constexpr bool value = true; };

template <class T>
__global__ void k_cfl_rate(Geo<T> g, F8<T> x, const double* ich, const double* vv, const double* ih, double gamma,
                           double whistler, double* partial) {
    int jj = blockIdx.y, k = blockIdx.z;
    double best = 0.0;
    const int nx = g.mx;
    const double* ichx = ich;
    const double* ichy = ich + nx;
    const double* ichz = ich + nx + g.my;
    const double* vvx = vv;
    const double* vvy = vv + nx;
    const double* vvz = vv + nx + g.my;
    const double* ihx = ih;
    const double* ihy = ih + nx;
    const double* ihz = ih + nx + g.my;
    if (k >= g.kcfl0 && k <= g.mz - 3 && jj <= g.my - 2) {
        const double r0 = g.rho0[k], bx0 = g.bx0[k], by0 = g.by0[k], bz0 = g.bz0[k], p0 = g.p0[k];
        const double cy = ichy[jj], vy_ = vvy[jj], cz = ichz[k], vz_ = vvz[k], hy = ihy[jj], hz = ihz[k];
        for (int i = threadIdx.x; i <= g.mx - 3; i += blockDim.x) {
            long c = (long)i + (long)jj * g.sy + (long)k * g.sz;
            best = nanmax(best, cfl_node_rate(x, c, r0, bx0, by0, bz0, p0, gamma, whistler, ichx[i], vvx[i], ihx[i],
                                              cy, vy_, hy, cz, vz_, hz));
        }
    }
    __shared__ double sh[32];
    double v = best;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = nanmax(v, __shfl_down_sync(0xffffffffu, v, o));
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    if (wid == 0) {
        int nw = (blockDim.x + 31) >> 5;
        v = lane < nw ? sh[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = nanmax(v, __shfl_down_sync(0xffffffffu, v, o));
        if (lane == 0) partial[(long)blockIdx.z * gridDim.y + blockIdx.y] = v;
    }
}

// dt = min(100, 1 / max rate) from the row partials, one block, fixed order
static __global__ void k_reduce_rate(const double* partial, long n, double* out) {
    double v = 0.0;
    for (long q = threadIdx.x; q < n; q += blockDim.x) v = nanmax(v, partial[q]);
    __shared__ double sh[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = nanmax(v, __shfl_down_sync(0xffffffffu, v, o));
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    if (wid == 0) {
        int nw = (blockDim.x + 31) >> 5;
        v = lane < nw ? sh[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = nanmax(v, __shfl_down_sync(0xffffffffu, v, o));
        if (lane == 0) *out = (v != v) ? v : fmin(100.0, 1.0 / v);
    }
}


// Diagnostics partial sums per (j,k) row: mass, energy (trapezoid weights), and the
// per-row extrema of J on the mid-y plane; partial layout [row][5]: mass, energy, jmax/jmin
// handled separately.  Planes klo..khi count (a z-slab's own planes and the walls it holds);
// the others give zero.
template <class T>
__global__ void k_diag_rows(Geo<T> g, F8<T> x, const double* wx, const double* wy, const double* wz,
                            double gamma, double* part, int klo, int khi) {
    int jj = blockIdx.y, k = blockIdx.z;
    if (k < klo || k > khi) {
        if (threadIdx.x == 0) {
            long row = (long)k * gridDim.y + jj;
            part[2 * row] = 0.;
            part[2 * row + 1] = 0.;
        }
        return;
    }
    const double r0 = g.rho0[k], bx0 = g.bx0[k], by0 = g.by0[k], bz0 = g.bz0[k], p0 = g.p0[k];
    double sm = 0., se = 0.;
    for (int i = threadIdx.x; i < g.mx; i += blockDim.x) {
        long c = (long)i + (long)jj * g.sy + (long)k * g.sz;
        double rho = r0 + (double)x.f[0][c];
        double m1 = x.f[1][c], m2 = x.f[2][c], m3 = x.f[3][c];
        double b1 = bx0 + (double)x.f[4][c], b2 = by0 + (double)x.f[5][c], b3 = bz0 + (double)x.f[6][c];
        double p = p0 + (double)x.f[7][c];
        double vol = wx[i];
        sm += rho * vol;
        se += (0.5 * (m1 * m1 + m2 * m2 + m3 * m3) / rho + p / (gamma - 1.) + 0.5 * (b1 * b1 + b2 * b2 + b3 * b3)) * vol;
    }
    __shared__ double s1[32], s2[32];
    sm = warp_sum(sm); se = warp_sum(se);
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) { s1[wid] = sm; s2[wid] = se; }
    __syncthreads();
    if (wid == 0) {
        int nw = (blockDim.x + 31) >> 5;
        sm = lane < nw ? s1[lane] : 0.;
        se = lane < nw ? s2[lane] : 0.;
        sm = warp_sum(sm); se = warp_sum(se);
        if (lane == 0) {
            long row = (long)k * gridDim.y + jj;
            part[2 * row] = sm * wy[jj] * wz[k];
            part[2 * row + 1] = se * wy[jj] * wz[k];
        }
    }
}

// Reconnected flux partials per y row (one block per j): sum_x sqrt(Bz(z=0)^2+eps^2)*wx, with
// Bz on the central plane ka (odd mz, kb = ka) or the mean of the two central planes ka, kb =
// ka + 1 (even mz); ka < 0: a z-slab that does not own the (first) central plane.
template <class T>
__global__ void k_diag_flux(Geo<T> g, F8<T> x, const double* wx, double* part, int ka, int kb) {
    int jj = blockIdx.x;
    double s = 0.;
    for (int i = threadIdx.x; i < g.mx && ka >= 0; i += blockDim.x) {
        double bz;
        if (ka == kb) {
            bz = g.bz0[ka] + (double)x.f[6][(long)i + (long)jj * g.sy + (long)ka * g.sz];
        } else {
            double za = g.bz0[ka] + (double)x.f[6][(long)i + (long)jj * g.sy + (long)ka * g.sz];
            double zb = g.bz0[kb] + (double)x.f[6][(long)i + (long)jj * g.sy + (long)kb * g.sz];
            bz = 0.5 * (za + zb);
        }
        s += sqrt(bz * bz + 1e-20) * wx[i];
    }
    __shared__ double sh[32];
    s = warp_sum(s);
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) sh[wid] = s;
    __syncthreads();
    if (wid == 0) {
        int nw = (blockDim.x + 31) >> 5;
        s = lane < nw ? sh[lane] : 0.;
        s = warp_sum(s);
        if (lane == 0) part[jj] = s;
    }
}

// J extrema on the mid-y plane (diagn t3dsdsc.f:1199-1214): one block per k row.
template <class T>
__global__ void k_diag_jext(Geo<T> g, F3<T> cur, int jm, double* part, int klo, int khi) {
    int k = blockIdx.x;
    double mx[3] = {-1e300, -1e300, -1e300}, mn[3] = {1e300, 1e300, 1e300};
    for (int i = threadIdx.x; i < g.mx && k >= klo && k <= khi; i += blockDim.x) {
        long c = (long)i + (long)jm * g.sy + (long)k * g.sz;
#pragma unroll
        for (int m = 0; m < 3; ++m) {
            double v = cur.f[m][c];
            mx[m] = fmax(mx[m], v);
            mn[m] = fmin(mn[m], v);
        }
    }
    __shared__ double sh[6][32];
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int m = 0; m < 3; ++m) {
        double a = warp_max(mx[m]), b = warp_min(mn[m]);
        if (lane == 0) { sh[2 * m][wid] = a; sh[2 * m + 1][wid] = b; }
    }
    __syncthreads();
    if (wid == 0) {
        int nw = (blockDim.x + 31) >> 5;
#pragma unroll
        for (int m = 0; m < 3; ++m) {
            double a = lane < nw ? sh[2 * m][lane] : -1e300;
            double b = lane < nw ? sh[2 * m + 1][lane] : 1e300;
            a = warp_max(a); b = warp_min(b);
            if (lane == 0) { part[6 * k + 2 * m] = a; part[6 * k + 2 * m + 1] = b; }
        }
    }
}

// Final diagnostics reduction (one block, fixed order) -> out[9]; also raises the blow-up
// flag when max Jy >= 1e7 (t3dsdsc.f:1232).
static __global__ void k_diag_final(const double* rows, long nrows, const double* fl, int my, const double* jext, int mz,
                             double* out, int* blowup) {
    __shared__ double sh[2][32];
    double sm = 0., se = 0.;
    for (long q = threadIdx.x; q < nrows; q += blockDim.x) { sm += rows[2 * q]; se += rows[2 * q + 1]; }
    sm = warp_sum(sm); se = warp_sum(se);
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) { sh[0][wid] = sm; sh[1][wid] = se; }
    __syncthreads();
    if (threadIdx.x == 0) {
        int nw = (blockDim.x + 31) >> 5;
        double a = 0., b = 0.;
        for (int w = 0; w < nw; ++w) { a += sh[0][w]; b += sh[1][w]; }
        double f = 0.;
        for (int j = 0; j < my; ++j) f += fl[j];
        double e[6] = {-1e300, 1e300, -1e300, 1e300, -1e300, 1e300};
        for (int k = 0; k < mz; ++k)
            for (int m = 0; m < 3; ++m) {
                e[2 * m] = fmax(e[2 * m], jext[6 * k + 2 * m]);
                e[2 * m + 1] = fmin(e[2 * m + 1], jext[6 * k + 2 * m + 1]);
            }
        out[0] = a; out[1] = b; out[2] = f / my;
        for (int q = 0; q < 6; ++q) out[3 + q] = e[q];
        if (blowup && (fabs(e[2]) >= 1e7 || e[2] != e[2])) *blowup = 1;
    }
}

}  // namespace dasha
