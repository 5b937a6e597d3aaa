// k_zhydro: the hydro part of the right-hand side (right, t3dsdsc.f:1334-1566 with bndry):
// continuity, momentum (fluxes rho v_i v_j + (p - p0) delta_ij, J x B - xresd) and the pressure
// equation, for the case without viscosity and diffusion; z-marching and register-blocked.
//
// A warp covers 32*VX consecutive x nodes (VX = 2 in FP32: float pairs), one row per warp, TY
// warps per CTA.  Planes of m1, m2, m3, p - p0 and rho - rho0 (tile plus a 2-node x/y halo, no
// corners) stream into an NS = D + 5 stage shared-memory ring with cp.async; the thread whose
// copy landed turns rho - rho0 into 1/rho in place.  The five quantities of the own nodes for
// planes c-2 .. c+2 stay in a register queue (the z stencil), so per plane a thread reads plane
// c+2 of its nodes, the x neighbours beyond its pair and rows c+-1, c+-2.  Fluxes are formed at
// each stencil node from (m, p - p0, 1/rho) there, as in the reference (m_i m_d / rho as
// m_i v_d with v_d = m_d / rho formed once per node).  At step c the ring is
// read at planes c and c+2, and by threads one step behind at c-1 and c+1; the first step also
// reads planes c-2 .. c+1 for the queue, so it holds planes c-2 .. c+2+D (hence D + 5 stages),
// and ends with a second barrier.
//
// TMA (k_zhydro_tma; not built with -DDASHA_NO_TMA): a CTA whose ring box (x0-OFF .. x0+TX+OFF-1,
// rows y0-2 .. y0+TY+1) lies inside the grid loads each ring plane as 5 `cp.async.bulk.tensor`
// boxes of exactly the ring plane's layout, issued by thread 0 against one mbarrier per stage;
// every thread waits on the stage's mbarrier (time-bounded: after about a second the kernel
// records g_wait_timeout, waits, again bounded, for the boxes it issued and returns) and turns
// its share of the plane's rho - rho0 into 1/rho before the plane's barrier.  CTAs whose halo
// wraps around x or y keep the cp.async element copies (a box cannot wrap).  The compute is the
// same code in both kernels; the engine picks one.
#pragma once

#include <type_traits>

#include "tma.cuh"

namespace dasha {

// the five ring fields (m1 m2 m3 dp drho) as 3-D tensor maps with the box of one ring plane
struct ZhMaps { CUtensorMap m[5]; };

template <class T, int VX, int TY, int D>
struct ZH {
    static constexpr int TX = 32 * VX;
    static constexpr int EPC = 16 / (int)sizeof(T);
    static constexpr int OFF = EPC;                   // interior column offset (>= 2)
    static constexpr int RS = TX + 2 * OFF;
    static constexpr int NR = TY + 4;                 // rows y0-2 .. y0+TY+1
    static constexpr int SP = NR * RS;
    static constexpr int NF = 5;                      // m1 m2 m3 dp ri
    static constexpr int NS = D + 5;
    static constexpr int CH = TX / EPC;
    static constexpr size_t smem() { return sizeof(T) * (size_t)NS * NF * SP; }
    // k_zhydro_tma: the ring 128-byte aligned, then one mbarrier per stage
    static constexpr size_t smem_tma() { return 128 + smem() + 8 * NS; }
};

// out: xdif 0 (rho), 1..3 (m), 4 (p); src: rho-rho0, m1, m2, m3, p-p0; pointwise J, B
template <class T>
struct HydroIO {
    const T *drho, *m1, *m2, *m3, *dp;
    const T *j1, *j2, *j3, *b1, *b2, *b3;
    T* out[5];
};

template <class T, int VX, int TY, int D, bool TMA>
__device__ __forceinline__ void zhydro_body(const Geo<T>& g, const HydroIO<T>& io, int chunk, const ZhMaps* maps) {
    using Z = ZH<T, VX, TY, D>;
    constexpr int TX = Z::TX, EPC = Z::EPC, OFF = Z::OFF, RS = Z::RS, NR = Z::NR, SP = Z::SP, NF = Z::NF,
                  NS = Z::NS, CH = Z::CH;
    constexpr int NT = 32 * TY;
    constexpr int NVEC = NR * CH;
    constexpr int NHAL = 4 * TY;                      // x-halo columns x0-2, x0-1, x0+wx, x0+wx+1 on the tile rows
    using IO = VIO<T, VX>;
    extern __shared__ __align__(16) unsigned char zh_smem_raw[];
    unsigned char* sbase = zh_smem_raw;
    if constexpr (TMA) sbase += (128 - (smem_addr(zh_smem_raw) & 127)) & 127;
    T* ring = reinterpret_cast<T*>(sbase);            // [NS][NF][SP]: m1 m2 m3 dp ri
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const int wx = min(TX, g.mx - x0);
    const int mz = g.mz;
    const int k0 = blockIdx.z * chunk;
    const int k1 = min(k0 + chunk, mz);
    const int cA = max(k0, 2), cB = min(k1 - 1, mz - 3);
    if (cA > cB) return;
    // a CTA whose ring box lies inside the grid loads it by TMA (k_zhydro_tma)
    const bool tma = TMA && x0 >= OFF && x0 + TX + OFF <= g.mx && y0 >= 2 && y0 + TY + 2 <= g.my;
    unsigned long long* bars = reinterpret_cast<unsigned long long*>(ring + (size_t)NS * NF * SP);
#ifndef DASHA_NO_TMA
    if constexpr (TMA) {
        if (tid == 0)
            for (int q = 0; q < NS; ++q) mbar_init(bars + q, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        __syncthreads();
    }
#endif
    const T* srcf[NF] = {io.m1, io.m2, io.m3, io.dp, io.drho};
    constexpr int NSL = (NVEC + NHAL + NT - 1) / NT;
    long gsrc[NSL];
    int sdst[NSL];
    bool svec[NSL];
#pragma unroll
    for (int q = 0; q < NSL; ++q) {
        const int sl = tid + q * NT;
        gsrc[q] = -1;
        sdst[q] = 0;
        svec[q] = sl < NVEC;
        if (sl < NVEC) {
            const int r = sl / CH, ch = sl % CH;
            if (ch * EPC < wx) {
                gsrc[q] = (long)(x0 + ch * EPC) + (long)pmod(y0 - 2 + r, g.my) * g.sy;
                sdst[q] = r * RS + OFF + ch * EPC;
            }
        } else if (sl < NVEC + NHAL) {
            const int h = sl - NVEC, r = h % TY + 2, side = h / TY;   // side 0..3: x0-2, x0-1, x0+wx, x0+wx+1
            const int dx = side < 2 ? side - 2 : wx + side - 2;
            gsrc[q] = (long)pmod(x0 + dx, g.mx) + (long)pmod(y0 - 2 + r, g.my) * g.sy;
            sdst[q] = r * RS + OFF + dx;
        }
    }
    const int phi = cB + 2;
    auto issue = [&](int p) {
#ifndef DASHA_NO_TMA
        if (tma) {
            if (tid == 0 && p <= phi) {
                T* stg = ring + (size_t)(p % NS) * NF * SP;
                unsigned long long* bar = bars + p % NS;
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // after the stage's generic accesses
                mbar_expect_tx(bar, (unsigned)(NF * SP * sizeof(T)));
#pragma unroll
                for (int f = 0; f < NF; ++f) tma_load_3d(stg + f * SP, &maps->m[f], x0 - OFF, y0 - 2, p, bar);
            }
            return;
        }
#else
        (void)bars;
        (void)maps;
#endif
        if (p <= phi) {
            T* stg = ring + (size_t)(p % NS) * NF * SP;
#pragma unroll
            for (int q = 0; q < NSL; ++q) {
                if (gsrc[q] >= 0) {
                    const long zo = gsrc[q] + (long)p * g.sz;
                    if (!DASHA_SPAN(zo, svec[q] ? EPC : 1, g.sz * (long)g.mz, BS_ZHYDRO_LOAD)) continue;
#pragma unroll
                    for (int f = 0; f < NF; ++f) {
                        if (svec[q]) cp_async16(stg + f * SP + sdst[q], srcf[f] + zo);
                        else cp_async_elem(stg + f * SP + sdst[q], srcf[f] + zo);
                    }
                }
            }
        }
        cp_async_commit();
    };
    // 1/rho of the nodes this thread copied in plane p (its own copies have landed)
    auto make_ri = [&](int p) {
        const T r0 = T(g.rho0[p]);
        T* ri = ring + (size_t)(p % NS) * NF * SP + 4 * SP;
#pragma unroll
        for (int q = 0; q < NSL; ++q) {
            if (gsrc[q] >= 0) {
                if (svec[q]) {
#pragma unroll
                    for (int e = 0; e < EPC; ++e) ri[sdst[q] + e] = recip(r0 + ri[sdst[q] + e]);
                } else {
                    ri[sdst[q]] = recip(r0 + ri[sdst[q]]);
                }
            }
        }
    };
#pragma unroll
    for (int p = 0; p < D + 4; ++p) issue(cA - 2 + p);   // planes cA-2 .. cA+1+D

    const int xl = VX * lane;
    const bool xon = xl < wx;
    const int gi = x0 + (xon ? xl : 0);
    const int gj = y0 + w;
    const bool yon = gj < g.my;
    const int jj = yon ? gj : g.my - 1;
    T ax[VX], bx[VX], cx[VX], dx[VX];
#pragma unroll
    for (int e = 0; e < VX; ++e) { ax[e] = g.a1x[gi + e]; bx[e] = g.b1x[gi + e]; cx[e] = g.c1x[gi + e]; dx[e] = g.d1x[gi + e]; }
    const T ay = g.a1y[jj], by = g.b1y[jj], cy = g.c1y[jj], dy = g.d1y[jj];
    const int me = (w + 2) * RS + OFF + xl;           // own first node in a ring plane
    const long col = (long)gi + (long)jj * g.sy;
    T zq[5][NF][VX];                                  // own (m1 m2 m3 dp ri), planes c-2 .. c+2
    bool primed = false;
    for (int c = cA; c <= cB; ++c) {
        issue(c + 2 + D);
        // pointwise operands of plane c, loaded before the barrier
        T j1[VX], j2[VX], j3[VX], b1[VX], b2[VX], b3[VX];
        if (xon && yon && DASHA_SPAN(col + (long)c * g.sz, VX, g.sz * (long)g.mz, BS_ZHYDRO_NODE_LOAD)) {
            const long q = col + (long)c * g.sz;
            IO::ld(io.j1 + q, j1); IO::ld(io.j2 + q, j2); IO::ld(io.j3 + q, j3);
            IO::ld(io.b1 + q, b1); IO::ld(io.b2 + q, b2); IO::ld(io.b3 + q, b3);
        }
        const T az = g.a1z[c], bz = g.b1z[c], cz = g.c1z[c], dz = g.d1z[c];
#ifndef DASHA_NO_TMA
        if (tma) {
            // planes c-2 .. c+2 on the first step, then c+2: wait, then 1/rho over the plane
            bool late = false;
            for (int p = primed ? c + 2 : c - 2; p <= c + 2; ++p) {
                if (!mbar_wait_bounded(bars + p % NS, (unsigned)(((p - (cA - 2)) / NS) & 1))) { late = true; break; }
                const T r0 = T(g.rho0[p]);
                T* ri = ring + (size_t)(p % NS) * NF * SP + 4 * SP;
                for (int i = tid; i < SP; i += NT) ri[i] = recip(r0 + ri[i]);
            }
            // these generic writes precede the boxes that refill the stage later
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            if (__syncthreads_or(late)) {
                // every box issued so far (planes up to c+2+D) lands before the CTA leaves
                if (tid == 0) atomicExch(&g_wait_timeout, 1u);
                for (int p = c - 2; p <= min(c + 2 + D, phi); ++p) {
                    if (p < cA - 2) continue;
                    mbar_wait_bounded(bars + p % NS, (unsigned)(((p - (cA - 2)) / NS) & 1));
                }
                return;
            }
        } else
#endif
        {
            cp_async_wait<D>();
            if (!primed)
                for (int p = c - 2; p <= c + 2; ++p) make_ri(p);
            else
                make_ri(c + 2);
            __syncthreads();
        }
        const T* pc = ring + (size_t)(c % NS) * NF * SP;
        if (!primed) {
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                const T* ps = ring + (size_t)((c - 2 + s) % NS) * NF * SP;
#pragma unroll
                for (int f = 0; f < NF; ++f) IO::ld(ps + f * SP + me, zq[s][f]);
            }
            primed = true;
            __syncthreads();   // planes c-2, c-1 are refilled within the next steps
        }
        {
            const T* p2 = ring + (size_t)((c + 2) % NS) * NF * SP;
#pragma unroll
            for (int f = 0; f < NF; ++f) IO::ld(p2 + f * SP + me, zq[4][f]);
        }
        if (xon && yon) {
            // o[0..4]: xdif of rho, m1, m2, m3, p; dv = -div(v) terms; grad p
            T o[5][VX], dvv[VX], px[VX], py[VX], pz[VX];
            // the six x/y/z quantities of one stencil node from (m1 m2 m3 dp ri) there:
            // direction d: m_d, F_1d, F_2d, F_3d (+ dp on the diagonal), dp, v_d
            if constexpr (std::is_same<T, float>::value && VX == 1) {
            // FP32, one node per thread: the six quantities of a direction as three packed pairs,
            // each five-point derivative of a pair one FMUL2 + three FFMA2 after four FADD2
            auto d1p = [](const float2 (&q)[5], float2 a2, float2 b2, float2 c2, float2 d2) {
                return d1fc2(q[0], q[1], q[2], q[3], q[4], a2, b2, c2, d2);
            };
            // ---- x: pairs (m1, m1 v1 + dp), (m2 v1, m3 v1), (dp, v1) ----
            {
                float2 P0[5], P1[5], P2[5];
#pragma unroll
                for (int s2 = 0; s2 < 5; ++s2) {
                    const int off = s2 - 2;
                    float v[NF];
#pragma unroll
                    for (int f = 0; f < NF; ++f) v[f] = off == 0 ? zq[2][f][0] : pc[f * SP + me + off];
                    const float a = v[0] * v[4];
                    P0[s2] = make_float2(v[0], fmaf(v[0], a, v[3]));
                    P1[s2] = __fmul2_rn(make_float2(v[1], v[2]), make_float2(a, a));
                    P2[s2] = make_float2(v[3], a);
                }
                const float2 A2 = make_float2(ax[0], ax[0]), B2 = make_float2(bx[0], bx[0]);
                const float2 C2 = make_float2(cx[0], cx[0]), D2 = make_float2(dx[0], dx[0]);
                const float2 r0 = d1p(P0, A2, B2, C2, D2), r1 = d1p(P1, A2, B2, C2, D2), r2 = d1p(P2, A2, B2, C2, D2);
                o[0][0] = -r0.x; o[1][0] = -r0.y; o[2][0] = -r1.x; o[3][0] = -r1.y;
                px[0] = r2.x; dvv[0] = -r2.y;
            }
            // ---- y: pairs (m2, m2 v2 + dp), (m1 v2, m3 v2), (dp, v2) ----
            {
                float2 P0[5], P1[5], P2[5];
#pragma unroll
                for (int s2 = 0; s2 < 5; ++s2) {
                    const int off = s2 - 2;
                    float v[NF];
#pragma unroll
                    for (int f = 0; f < NF; ++f) v[f] = off == 0 ? zq[2][f][0] : pc[f * SP + me + off * RS];
                    const float b = v[1] * v[4];
                    P0[s2] = make_float2(v[1], fmaf(v[1], b, v[3]));
                    P1[s2] = __fmul2_rn(make_float2(v[0], v[2]), make_float2(b, b));
                    P2[s2] = make_float2(v[3], b);
                }
                const float2 A2 = make_float2(ay, ay), B2 = make_float2(by, by), C2 = make_float2(cy, cy), D2 = make_float2(dy, dy);
                const float2 r0 = d1p(P0, A2, B2, C2, D2), r1 = d1p(P1, A2, B2, C2, D2), r2 = d1p(P2, A2, B2, C2, D2);
                o[0][0] -= r0.x; o[2][0] -= r0.y; o[1][0] -= r1.x; o[3][0] -= r1.y;
                py[0] = r2.x; dvv[0] -= r2.y;
            }
            // ---- z: pairs (m3, m3 v3 + dp), (m1 v3, m2 v3), (dp, v3), from the register queue ----
            {
                float2 P0[5], P1[5], P2[5];
#pragma unroll
                for (int s2 = 0; s2 < 5; ++s2) {
                    const float m1 = zq[s2][0][0], m2 = zq[s2][1][0], m3 = zq[s2][2][0], dp = zq[s2][3][0], ri = zq[s2][4][0];
                    const float v3 = m3 * ri;
                    P0[s2] = make_float2(m3, fmaf(m3, v3, dp));
                    P1[s2] = __fmul2_rn(make_float2(m1, m2), make_float2(v3, v3));
                    P2[s2] = make_float2(dp, v3);
                }
                const float2 A2 = make_float2(az, az), B2 = make_float2(bz, bz), C2 = make_float2(cz, cz), D2 = make_float2(dz, dz);
                const float2 r0 = d1p(P0, A2, B2, C2, D2), r1 = d1p(P1, A2, B2, C2, D2), r2 = d1p(P2, A2, B2, C2, D2);
                o[0][0] -= r0.x; o[3][0] -= r0.y; o[1][0] -= r1.x; o[2][0] -= r1.y;
                pz[0] = r2.x + T(g.dzp0[c]); dvv[0] -= r2.y;
            }
            } else {
            // ---- x ----
            {
                T lo[NF][2], hi[NF][2];
#pragma unroll
                for (int f = 0; f < NF; ++f) {
                    lo[f][0] = pc[f * SP + me - 2]; lo[f][1] = pc[f * SP + me - 1];
                    hi[f][0] = pc[f * SP + me + VX]; hi[f][1] = pc[f * SP + me + VX + 1];
                }
                // the six quantities at the VX + 4 x nodes -2 .. VX+1, each formed once for the
                // VX stencils that share it
                T q6[6][VX + 4];
#pragma unroll
                for (int k = -2; k < VX + 2; ++k) {
                    T v[NF];
#pragma unroll
                    for (int f = 0; f < NF; ++f)
                        v[f] = k < 0 ? lo[f][k + 2] : (k >= VX ? hi[f][k - VX] : zq[2][f][k < 0 ? 0 : (k >= VX ? VX - 1 : k)]);
                    const T a = v[0] * v[4];                 // v1
                    q6[0][k + 2] = v[0];
                    q6[1][k + 2] = v[0] * a + v[3];
                    q6[2][k + 2] = v[1] * a;
                    q6[3][k + 2] = v[2] * a;
                    q6[4][k + 2] = v[3];
                    q6[5][k + 2] = a;
                }
#pragma unroll
                for (int e = 0; e < VX; ++e) {
                    T dd[6];
#pragma unroll
                    for (int u = 0; u < 6; ++u)
                        dd[u] = d1fc(q6[u][e], q6[u][e + 1], q6[u][e + 2], q6[u][e + 3], q6[u][e + 4], ax[e], bx[e], cx[e], dx[e]);
                    o[0][e] = -dd[0]; o[1][e] = -dd[1]; o[2][e] = -dd[2]; o[3][e] = -dd[3];
                    px[e] = dd[4]; dvv[e] = -dd[5];
                }
            }
            // ---- y ----
            {
                T ym[2][NF][VX], yp[2][NF][VX];   // rows -2, -1 and +1, +2
#pragma unroll
                for (int f = 0; f < NF; ++f) {
                    IO::ld(pc + f * SP + me - 2 * RS, ym[0][f]); IO::ld(pc + f * SP + me - RS, ym[1][f]);
                    IO::ld(pc + f * SP + me + RS, yp[0][f]); IO::ld(pc + f * SP + me + 2 * RS, yp[1][f]);
                }
#pragma unroll
                for (int e = 0; e < VX; ++e) {
                    T q6[6][5];
#pragma unroll
                    for (int s = 0; s < 5; ++s) {
                        T v[NF];
#pragma unroll
                        for (int f = 0; f < NF; ++f)
                            v[f] = s < 2 ? ym[s][f][e] : (s == 2 ? zq[2][f][e] : yp[s - 3 < 0 ? 0 : s - 3][f][e]);
                        const T b = v[1] * v[4];                 // v2
                        q6[0][s] = v[1];
                        q6[1][s] = v[0] * b;
                        q6[2][s] = v[1] * b + v[3];
                        q6[3][s] = v[2] * b;
                        q6[4][s] = v[3];
                        q6[5][s] = b;
                    }
                    T dd[6];
#pragma unroll
                    for (int u = 0; u < 6; ++u) dd[u] = d1fc(q6[u][0], q6[u][1], q6[u][2], q6[u][3], q6[u][4], ay, by, cy, dy);
                    o[0][e] -= dd[0]; o[1][e] -= dd[1]; o[2][e] -= dd[2]; o[3][e] -= dd[3];
                    py[e] = dd[4]; dvv[e] -= dd[5];
                }
            }
            // ---- z ----
#pragma unroll
            for (int e = 0; e < VX; ++e) {
                T q6[6][5];
#pragma unroll
                for (int s = 0; s < 5; ++s) {
                    const T m1 = zq[s][0][e], m2 = zq[s][1][e], m3 = zq[s][2][e], dp = zq[s][3][e], ri = zq[s][4][e];
                    const T v3 = m3 * ri;
                    q6[0][s] = m3;
                    q6[1][s] = m1 * v3;
                    q6[2][s] = m2 * v3;
                    q6[3][s] = m3 * v3 + dp;
                    q6[4][s] = dp;
                    q6[5][s] = v3;
                }
                T dd[6];
#pragma unroll
                for (int u = 0; u < 6; ++u) dd[u] = d1fc(q6[u][0], q6[u][1], q6[u][2], q6[u][3], q6[u][4], az, bz, cz, dz);
                o[0][e] -= dd[0]; o[1][e] -= dd[1]; o[2][e] -= dd[2]; o[3][e] -= dd[3];
                pz[e] = dd[4] + T(g.dzp0[c]); dvv[e] -= dd[5];
            }
            }
            // ---- pointwise: J x B - xresd, pressure equation ----
            const T rsx = T(g.rsx[c]), rsy = T(g.rsy[c]), rsz = T(g.rsz[c]), p0 = T(g.p0[c]);
            const T bx0 = T(g.bx0[c]), by0 = T(g.by0[c]), bz0 = T(g.bz0[c]);
#pragma unroll
            for (int e = 0; e < VX; ++e) {
                const T B1 = bx0 + b1[e], B2 = by0 + b2[e], B3 = bz0 + b3[e];
                o[1][e] = o[1][e] - rsx + j2[e] * B3 - j3[e] * B2;
                o[2][e] = o[2][e] - rsy + j3[e] * B1 - j1[e] * B3;
                o[3][e] = o[3][e] - rsz + j1[e] * B2 - j2[e] * B1;
                const T ri = zq[2][4][e];
                const T v1 = zq[2][0][e] * ri, v2 = zq[2][1][e] * ri, v3 = zq[2][2][e] * ri;
                const T pcn = p0 + zq[2][3][e];
                o[4][e] = -px[e] * v1 - py[e] * v2 - pz[e] * v3 + dvv[e] * g.gamma * pcn +
                          (g.gamma - T(1)) * g.eta * (j1[e] * j1[e] + j2[e] * j2[e] + j3[e] * j3[e]);
            }
#pragma unroll
            for (int m = 0; m < 5; ++m)
                if (DASHA_SPAN(col + (long)c * g.sz, VX, g.sz * (long)g.mz, BS_ZHYDRO_STORE)) IO::st(io.out[m] + col + (long)c * g.sz, o[m]);
            if (c == 2 || c == mz - 3) {
                const int kh = c == 2 ? 1 : mz - 2, kz = c == 2 ? 0 : mz - 1;
#pragma unroll
                for (int m = 0; m < 5; ++m) {
                    T hv[VX], zv[VX];
#pragma unroll
                    for (int e = 0; e < VX; ++e) { hv[e] = T(0.5) * o[m][e]; zv[e] = T(0); }
                    IO::st(io.out[m] + col + (long)kh * g.sz, hv);
                    IO::st(io.out[m] + col + (long)kz * g.sz, zv);
                }
            }
        }
#pragma unroll
        for (int s = 0; s < 4; ++s)
#pragma unroll
            for (int f = 0; f < NF; ++f)
#pragma unroll
                for (int e = 0; e < VX; ++e) zq[s][f][e] = zq[s + 1][f][e];
    }
    cp_async_wait<0>();
}

template <class T, int VX, int TY, int D, int MINB = 1>
__global__ void __launch_bounds__(32 * TY, MINB) k_zhydro(Geo<T> g, HydroIO<T> io, int chunk) {
    zhydro_body<T, VX, TY, D, false>(g, io, chunk, nullptr);
}

#ifndef DASHA_NO_TMA
template <class T, int VX, int TY, int D, int MINB = 1>
__global__ void __launch_bounds__(32 * TY, MINB) k_zhydro_tma(Geo<T> g, HydroIO<T> io, int chunk,
                                                              const __grid_constant__ ZhMaps maps) {
    zhydro_body<T, VX, TY, D, true>(g, io, chunk, &maps);
}
#endif

}  // namespace dasha
