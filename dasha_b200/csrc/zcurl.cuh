// k_zcurl: SIGN * curl of three fields with the 4th-order first derivatives of the stretched
// grid and the wall rows of the result, z-marching and register-blocked: SIGN = +1 is
// J1 = curl(B - B0) (current, t3dsdsc.f:2476-2491, with bndryc), SIGN = -1 is dB/dt = -curl E
// (induction, t3dsdsc.f:1435-1452).
//
// A warp covers 32*VX consecutive x nodes (VX = 2 in FP32: float pairs), one row per warp, TY
// warps per CTA.  Planes of the tile plus a 2-node x/y halo (no corners) stream into an
// NS = D + 5 stage shared-memory ring with cp.async.  The z derivatives need fields 0 and 1
// only: their own values for planes c-2 .. c+2 stay in a register queue, filled from the ring
// when plane c+2 lands, so per plane a thread reads plane c+2 of its nodes, the x neighbours
// beyond its pair (two 2-element loads per field) and the rows c+-1, c+-2 of fields 0 and 2.
// At step c the ring is read at planes c and c+2, and by threads one step behind at c-1 and
// c+1; the stage refilled at step c (plane c+2+D, NS = D + 5 stages) is none of them.  The
// first step also reads planes c-2 .. c+1 for the queue, so it holds planes c-2 .. c+2+D at
// once (hence D + 5 stages) and ends with a second barrier.
#pragma once

#include <type_traits>

namespace dasha {

template <class T, int VX, int TY, int D>
struct ZC3 {
    static constexpr int TX = 32 * VX;
    static constexpr int EPC = 16 / (int)sizeof(T);
    static constexpr int OFF = EPC;                   // interior column offset (>= 2)
    static constexpr int RS = TX + 2 * OFF;
    static constexpr int NR = TY + 4;                 // rows y0-2 .. y0+TY+1
    static constexpr int SP = NR * RS;
    static constexpr int NS = D + 5;                  // the first step holds planes c-2 .. c+2+D
    static constexpr int CH = TX / EPC;
    static constexpr size_t smem() { return sizeof(T) * (size_t)NS * 3 * SP; }
};

template <class T, int VX, int TY, int D, int SIGN>
__global__ void __launch_bounds__(32 * TY) k_zcurl(Geo<T> g, SrcFields<T, 3> src, F3<T> out, int chunk) {
    using Z = ZC3<T, VX, TY, D>;
    constexpr int TX = Z::TX, EPC = Z::EPC, OFF = Z::OFF, RS = Z::RS, NR = Z::NR, SP = Z::SP, NS = Z::NS, CH = Z::CH;
    constexpr int NT = 32 * TY;
    constexpr int NVEC = NR * CH;
    constexpr int NHAL = 4 * TY;                      // x-halo columns x0-2, x0-1, x0+wx, x0+wx+1 on the tile rows
    using IO = VIO<T, VX>;
    extern __shared__ __align__(16) unsigned char zc_smem_raw[];
    T* ring = reinterpret_cast<T*>(zc_smem_raw);      // [NS][3][SP]
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const int wx = min(TX, g.mx - x0);
    const int mz = g.mz;
    const int k0 = blockIdx.z * chunk;
    const int k1 = min(k0 + chunk, mz);
    const int cA = max(k0, 2), cB = min(k1 - 1, mz - 3);
    if (cA > cB) return;
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
        if (p <= phi) {
            T* stg = ring + (size_t)(p % NS) * 3 * SP;
#pragma unroll
            for (int q = 0; q < NSL; ++q) {
                if (gsrc[q] >= 0) {
                    const long zo = gsrc[q] + (long)p * g.sz;
                    if (!DASHA_SPAN(zo, svec[q] ? EPC : 1, g.sz * (long)g.mz, BS_ZCURL_LOAD)) continue;
#pragma unroll
                    for (int f = 0; f < 3; ++f) {
                        if (svec[q]) cp_async16(stg + f * SP + sdst[q], src.f[f] + zo);
                        else cp_async_elem(stg + f * SP + sdst[q], src.f[f] + zo);
                    }
                }
            }
        }
        cp_async_commit();
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
    // z queue of fields 0 and 1: planes c-2 .. c+2 (index 0 .. 4)
    T zq[5][2][VX];
    bool primed = false;
    for (int c = cA; c <= cB; ++c) {
        issue(c + 2 + D);
        const T az = g.a1z[c], bz = g.b1z[c], cz = g.c1z[c], dz = g.d1z[c];
        cp_async_wait<D>();
        __syncthreads();
        const T* pc = ring + (size_t)(c % NS) * 3 * SP;
        if (!primed) {
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                const T* ps = ring + (size_t)((c - 2 + s) % NS) * 3 * SP;
                IO::ld(ps + me, zq[s][0]);
                IO::ld(ps + SP + me, zq[s][1]);
            }
            primed = true;
            __syncthreads();   // planes c-2, c-1 are refilled within the next steps
        }
        {
            const T* p2 = ring + (size_t)((c + 2) % NS) * 3 * SP;
            IO::ld(p2 + me, zq[4][0]);
            IO::ld(p2 + SP + me, zq[4][1]);
        }
        if (xon && yon) {
            // x neighbours beyond the pair (fields 1 and 2): x-2, x-1 and x+VX, x+VX+1
            T l1[2], r1[2], l2[2], r2[2], c2[VX], c1[VX];
            l1[0] = pc[SP + me - 2]; l1[1] = pc[SP + me - 1]; r1[0] = pc[SP + me + VX]; r1[1] = pc[SP + me + VX + 1];
            l2[0] = pc[2 * SP + me - 2]; l2[1] = pc[2 * SP + me - 1]; r2[0] = pc[2 * SP + me + VX]; r2[1] = pc[2 * SP + me + VX + 1];
            IO::ld(pc + 2 * SP + me, c2);
#pragma unroll
            for (int e = 0; e < VX; ++e) c1[e] = zq[2][1][e];
            // y neighbours (fields 0 and 2): rows -2, -1, +1, +2
            T y0m2[VX], y0m1[VX], y0p1[VX], y0p2[VX], y2m2[VX], y2m1[VX], y2p1[VX], y2p2[VX];
            IO::ld(pc + me - 2 * RS, y0m2); IO::ld(pc + me - RS, y0m1); IO::ld(pc + me + RS, y0p1); IO::ld(pc + me + 2 * RS, y0p2);
            IO::ld(pc + 2 * SP + me - 2 * RS, y2m2); IO::ld(pc + 2 * SP + me - RS, y2m1);
            IO::ld(pc + 2 * SP + me + RS, y2p1); IO::ld(pc + 2 * SP + me + 2 * RS, y2p2);
            // x stencil value of field f at own node e, offset s in -2..2
            auto xv = [&](const T (&cen)[VX], const T (&lo)[2], const T (&hi)[2], int e, int s) -> T {
                const int k = e + s;
                return k < 0 ? lo[k + 2] : (k >= VX ? hi[k - VX] : cen[k < 0 ? 0 : (k >= VX ? VX - 1 : k)]);
            };
            T o[3][VX];
            if constexpr (std::is_same<T, float>::value && VX == 2) {
                // the pair's six derivatives as packed pairs (node 0, node 1), the roundings of
                // the scalar form below
                const float2 AX = make_float2(ax[0], ax[1]), BX = make_float2(bx[0], bx[1]);
                const float2 CX = make_float2(cx[0], cx[1]), DX = make_float2(dx[0], dx[1]);
                auto v2 = [](const float (&a)[2]) { return make_float2(a[0], a[1]); };
                auto zp = [&](int s, int f) { return make_float2(zq[s][f][0], zq[s][f][1]); };
                const float2 d1x = d1fc2(v2(l1), make_float2(l1[1], c1[0]), v2(c1), make_float2(c1[1], r1[0]), v2(r1),
                                         AX, BX, CX, DX);
                const float2 d2x = d1fc2(v2(l2), make_float2(l2[1], c2[0]), v2(c2), make_float2(c2[1], r2[0]), v2(r2),
                                         AX, BX, CX, DX);
                const float2 d0y = d1fc2(v2(y0m2), v2(y0m1), zp(2, 0), v2(y0p1), v2(y0p2), bc2(ay), bc2(by), bc2(cy), bc2(dy));
                const float2 d2y = d1fc2(v2(y2m2), v2(y2m1), v2(c2), v2(y2p1), v2(y2p2), bc2(ay), bc2(by), bc2(cy), bc2(dy));
                const float2 d0z = d1fc2(zp(0, 0), zp(1, 0), zp(2, 0), zp(3, 0), zp(4, 0), bc2(az), bc2(bz), bc2(cz), bc2(dz));
                const float2 d1z = d1fc2(zp(0, 1), zp(1, 1), zp(2, 1), zp(3, 1), zp(4, 1), bc2(az), bc2(bz), bc2(cz), bc2(dz));
                float2 r0, r1v, r2v;
                if (SIGN > 0) {
                    r0 = __fadd2_rn(d2y, neg2(d1z)); r1v = __fadd2_rn(d0z, neg2(d2x)); r2v = __fadd2_rn(d1x, neg2(d0y));
                } else {
                    r0 = __fadd2_rn(neg2(d2y), d1z); r1v = __fadd2_rn(neg2(d0z), d2x); r2v = __fadd2_rn(neg2(d1x), d0y);
                }
                o[0][0] = r0.x; o[0][1] = r0.y; o[1][0] = r1v.x; o[1][1] = r1v.y; o[2][0] = r2v.x; o[2][1] = r2v.y;
            } else {
#pragma unroll
            for (int e = 0; e < VX; ++e) {
                const T d1x = d1fc(xv(c1, l1, r1, e, -2), xv(c1, l1, r1, e, -1), c1[e], xv(c1, l1, r1, e, 1),
                                   xv(c1, l1, r1, e, 2), ax[e], bx[e], cx[e], dx[e]);
                const T d2x = d1fc(xv(c2, l2, r2, e, -2), xv(c2, l2, r2, e, -1), c2[e], xv(c2, l2, r2, e, 1),
                                   xv(c2, l2, r2, e, 2), ax[e], bx[e], cx[e], dx[e]);
                const T d0y = d1fc(y0m2[e], y0m1[e], zq[2][0][e], y0p1[e], y0p2[e], ay, by, cy, dy);
                const T d2y = d1fc(y2m2[e], y2m1[e], c2[e], y2p1[e], y2p2[e], ay, by, cy, dy);
                const T d0z = d1fc(zq[0][0][e], zq[1][0][e], zq[2][0][e], zq[3][0][e], zq[4][0][e], az, bz, cz, dz);
                const T d1z = d1fc(zq[0][1][e], zq[1][1][e], zq[2][1][e], zq[3][1][e], zq[4][1][e], az, bz, cz, dz);
                if (SIGN > 0) {
                    o[0][e] = d2y - d1z;
                    o[1][e] = d0z - d2x;
                    o[2][e] = d1x - d0y;
                } else {
                    o[0][e] = -d2y + d1z;
                    o[1][e] = -d0z + d2x;
                    o[2][e] = -d1x + d0y;
                }
            }
            }
            const long col = (long)gi + (long)gj * g.sy;
#pragma unroll
            for (int m = 0; m < 3; ++m)
                if (DASHA_SPAN(col + (long)c * g.sz, VX, g.sz * (long)g.mz, BS_ZCURL_STORE)) IO::st(out.f[m] + col + (long)c * g.sz, o[m]);
            if (c == 2 || c == mz - 3) {
                const int kh = c == 2 ? 1 : mz - 2, kz = c == 2 ? 0 : mz - 1;
#pragma unroll
                for (int m = 0; m < 3; ++m) {
                    T hv[VX], zv[VX];
#pragma unroll
                    for (int e = 0; e < VX; ++e) { hv[e] = T(0.5) * o[m][e]; zv[e] = T(0); }
                    IO::st(out.f[m] + col + (long)kh * g.sz, hv);
                    IO::st(out.f[m] + col + (long)kz * g.sz, zv);
                }
            }
        }
#pragma unroll
        for (int s = 0; s < 4; ++s)
#pragma unroll
            for (int f = 0; f < 2; ++f)
#pragma unroll
                for (int e = 0; e < VX; ++e) zq[s][f][e] = zq[s + 1][f][e];
    }
    cp_async_wait<0>();
}

}  // namespace dasha
