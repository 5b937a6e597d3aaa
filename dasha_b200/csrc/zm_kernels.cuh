// zm_kernels.cuh -- z-marching (2.5-D) building blocks: each CTA owns an x-y tile of columns
// and streams through a chunk of z planes, keeping the planes a stencil needs in a
// shared-memory ring filled by cp.async.  Global memory is read once per plane (plus the x-y
// halo, which neighbouring CTAs read at about the same time and so mostly hits L2) and
// written once.  This file holds the shared helpers and the radius-2 ring framework k_zst2
// (hydro RHS); the smoothing passes are k_zpv / k_zpv2 (zpv.cuh, zpv2.cuh), the curls k_zcurl
// (zcurl.cuh).
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
// source field pointers of a z-marching launch
template <class T, int NF>
struct SrcFields {
    const T* f[NF];
    __device__ __forceinline__ void load(const Geo<T>&, long idx, int, T v[NF]) const {
#pragma unroll
        for (int q = 0; q < NF; ++q) v[q] = f[q][idx];
    }
};

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

// KINDS (2 bits per field): does any of the first nf fields use the radial coefficient
__host__ __device__ constexpr bool any_kind0(unsigned kinds, int nf) {
    for (int f = 0; f < nf; ++f)
        if (((kinds >> (2 * f)) & 3u) == 0u) return true;
    return false;
}

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
