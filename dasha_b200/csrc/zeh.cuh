// k_zeh: the two pointwise-in-the-state fields of the RHS in one z-march (read once):
//   E0 = -v x B + eta J at every node (t3dsdsc.f:1367-1372), and
//   the Hall field di (J x B - grad p) / rho on rows 2..mz-3, half of rows 2 / mz-3 on rows 1 /
//   mz-2, zero on rows 0 / mz-1 (t3dsdsc.f:1391-1423 with bndryh).
// grad p = grad(p - p0) + dp0/dz e_z; of -di dp0/dz / rho, the plane-uniform part -di dp0/dz /
// rho0 has an exactly zero discrete curl (the Hall passes keep it uniform in x and y) and is left
// out; the rest is di dp0/dz (rho - rho0) / (rho0 rho).  This keeps an O(1) field out of the FP32
// sum that forms E.
//
// A warp covers 32*VX consecutive x nodes (VX = 2 in FP32), one row per warp, TY warps per CTA.
// Only p - p0 is differentiated: its planes (tile plus a 2-node x/y halo, no corners) stream into
// an NS = D + 5 stage ring with cp.async and its own values for planes c-2 .. c+2 stay in a
// register queue; rho, m, B and J are read at the node, before the plane's barrier.  Ring reads
// and stage reuse as in k_zcurl.
#pragma once

namespace dasha {

template <class T, int VX, int TY, int D>
struct ZEH {
    static constexpr int TX = 32 * VX;
    static constexpr int EPC = 16 / (int)sizeof(T);
    static constexpr int OFF = EPC;                   // interior column offset (>= 2)
    static constexpr int RS = TX + 2 * OFF;
    static constexpr int NR = TY + 4;                 // rows y0-2 .. y0+TY+1
    static constexpr int SP = NR * RS;
    static constexpr int NS = D + 5;
    static constexpr int CH = TX / EPC;
    static constexpr size_t smem() { return sizeof(T) * (size_t)NS * SP; }
};

template <class T>
struct EHIO {
    const T *drho, *m1, *m2, *m3, *b1, *b2, *b3, *dp;
    const T *j1, *j2, *j3;
    T *e[3], *h[3];
};

template <class T, int VX, int TY, int D>
__global__ void __launch_bounds__(32 * TY) k_zeh(Geo<T> g, EHIO<T> io, int chunk) {
    using Z = ZEH<T, VX, TY, D>;
    constexpr int TX = Z::TX, EPC = Z::EPC, OFF = Z::OFF, RS = Z::RS, NR = Z::NR, SP = Z::SP, NS = Z::NS, CH = Z::CH;
    constexpr int NT = 32 * TY;
    constexpr int NVEC = NR * CH;
    constexpr int NHAL = 4 * TY;                      // x-halo columns x0-2, x0-1, x0+wx, x0+wx+1 on the tile rows
    using IO = VIO<T, VX>;
    extern __shared__ __align__(16) unsigned char zeh_smem_raw[];
    T* ring = reinterpret_cast<T*>(zeh_smem_raw);     // [NS][SP]: p - p0
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
            const int h = sl - NVEC, r = h % TY + 2, side = h / TY;
            const int dx = side < 2 ? side - 2 : wx + side - 2;
            gsrc[q] = (long)pmod(x0 + dx, g.mx) + (long)pmod(y0 - 2 + r, g.my) * g.sy;
            sdst[q] = r * RS + OFF + dx;
        }
    }
    const int phi = cB + 2;
    auto issue = [&](int p) {
        if (p <= phi) {
            T* stg = ring + (size_t)(p % NS) * SP;
#pragma unroll
            for (int q = 0; q < NSL; ++q) {
                if (gsrc[q] >= 0 && DASHA_SPAN(gsrc[q] + (long)p * g.sz, svec[q] ? EPC : 1, g.sz * (long)g.mz, BS_ZEH_LOAD)) {
                    if (svec[q]) cp_async16(stg + sdst[q], io.dp + gsrc[q] + (long)p * g.sz);
                    else cp_async_elem(stg + sdst[q], io.dp + gsrc[q] + (long)p * g.sz);
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
    const bool act = xon && yon;
    const int jj = yon ? gj : g.my - 1;
    T ax[VX], bx[VX], cx[VX], dx[VX];
#pragma unroll
    for (int e = 0; e < VX; ++e) { ax[e] = g.a1x[gi + e]; bx[e] = g.b1x[gi + e]; cx[e] = g.c1x[gi + e]; dx[e] = g.d1x[gi + e]; }
    const T ay = g.a1y[jj], by = g.b1y[jj], cy = g.c1y[jj], dy = g.d1y[jj];
    const int me = (w + 2) * RS + OFF + xl;
    const long col = (long)gi + (long)jj * g.sy;
    // E0 at node index n of plane k from pointwise loads
    auto efield = [&](long n, int k, T (&e1)[VX], T (&e2)[VX], T (&e3)[VX]) {
        T dr[VX], a1[VX], a2[VX], a3[VX], c1[VX], c2[VX], c3[VX], q1[VX], q2[VX], q3[VX];
        IO::ld(io.drho + n, dr); IO::ld(io.m1 + n, a1); IO::ld(io.m2 + n, a2); IO::ld(io.m3 + n, a3);
        IO::ld(io.b1 + n, c1); IO::ld(io.b2 + n, c2); IO::ld(io.b3 + n, c3);
        IO::ld(io.j1 + n, q1); IO::ld(io.j2 + n, q2); IO::ld(io.j3 + n, q3);
        const T r0 = T(g.rho0[k]), bx0 = T(g.bx0[k]), by0 = T(g.by0[k]), bz0 = T(g.bz0[k]);
#pragma unroll
        for (int e = 0; e < VX; ++e) {
            const T ri = T(1) / (r0 + dr[e]);
            const T B1 = bx0 + c1[e], B2 = by0 + c2[e], B3 = bz0 + c3[e];
            e1[e] = (-a2[e] * B3 + a3[e] * B2) * ri + g.eta * q1[e];
            e2[e] = (-a3[e] * B1 + a1[e] * B3) * ri + g.eta * q2[e];
            e3[e] = (-a1[e] * B2 + a2[e] * B1) * ri + g.eta * q3[e];
        }
    };
    T zq[5][VX];                                      // own p - p0, planes c-2 .. c+2
    bool primed = false;
    for (int c = cA; c <= cB; ++c) {
        issue(c + 2 + D);
        T dr[VX], a1[VX], a2[VX], a3[VX], c1[VX], c2[VX], c3[VX], q1[VX], q2[VX], q3[VX];
        const long n = col + (long)c * g.sz;
        if (act) {
            IO::ld(io.drho + n, dr); IO::ld(io.m1 + n, a1); IO::ld(io.m2 + n, a2); IO::ld(io.m3 + n, a3);
            IO::ld(io.b1 + n, c1); IO::ld(io.b2 + n, c2); IO::ld(io.b3 + n, c3);
            IO::ld(io.j1 + n, q1); IO::ld(io.j2 + n, q2); IO::ld(io.j3 + n, q3);
        }
        const T az = g.a1z[c], bz = g.b1z[c], cz = g.c1z[c], dz = g.d1z[c];
        cp_async_wait<D>();
        __syncthreads();
        const T* pc = ring + (size_t)(c % NS) * SP;
        if (!primed) {
#pragma unroll
            for (int s = 0; s < 4; ++s) IO::ld(ring + (size_t)((c - 2 + s) % NS) * SP + me, zq[s]);
            primed = true;
            __syncthreads();   // planes c-2, c-1 are refilled within the next steps
        }
        IO::ld(ring + (size_t)((c + 2) % NS) * SP + me, zq[4]);
        if (act) {
            T l[2], h[2], ym2[VX], ym1[VX], yp1[VX], yp2[VX];
            l[0] = pc[me - 2]; l[1] = pc[me - 1]; h[0] = pc[me + VX]; h[1] = pc[me + VX + 1];
            IO::ld(pc + me - 2 * RS, ym2); IO::ld(pc + me - RS, ym1); IO::ld(pc + me + RS, yp1); IO::ld(pc + me + 2 * RS, yp2);
            const T r0 = T(g.rho0[c]), bx0 = T(g.bx0[c]), by0 = T(g.by0[c]), bz0 = T(g.bz0[c]), dzr = T(g.dzp0r[c]);
            T e1[VX], e2[VX], e3[VX], h1[VX], h2[VX], h3[VX];
#pragma unroll
            for (int e = 0; e < VX; ++e) {
                auto xv = [&](int s) -> T {
                    const int k = e + s;
                    return k < 0 ? l[k + 2] : (k >= VX ? h[k - VX] : zq[2][k < 0 ? 0 : (k >= VX ? VX - 1 : k)]);
                };
                const T px = d1fc(xv(-2), xv(-1), zq[2][e], xv(1), xv(2), ax[e], bx[e], cx[e], dx[e]);
                const T py = d1fc(ym2[e], ym1[e], zq[2][e], yp1[e], yp2[e], ay, by, cy, dy);
                const T pz = d1fc(zq[0][e], zq[1][e], zq[2][e], zq[3][e], zq[4][e], az, bz, cz, dz);
                const T r = r0 + dr[e];
                const T ri = T(1) / r;
                const T B1 = bx0 + c1[e], B2 = by0 + c2[e], B3 = bz0 + c3[e];
                e1[e] = (-a2[e] * B3 + a3[e] * B2) * ri + g.eta * q1[e];
                e2[e] = (-a3[e] * B1 + a1[e] * B3) * ri + g.eta * q2[e];
                e3[e] = (-a1[e] * B2 + a2[e] * B1) * ri + g.eta * q3[e];
                const T dir = g.di / r;
                h1[e] = (q2[e] * B3 - q3[e] * B2 - px) * dir;
                h2[e] = (q3[e] * B1 - q1[e] * B3 - py) * dir;
                h3[e] = (q1[e] * B2 - q2[e] * B1 - pz + dzr * dr[e]) * dir;
            }
            if (DASHA_SPAN(n, VX, g.sz * (long)g.mz, BS_ZEH_STORE)) { IO::st(io.e[0] + n, e1); IO::st(io.e[1] + n, e2); IO::st(io.e[2] + n, e3); }
            IO::st(io.h[0] + n, h1); IO::st(io.h[1] + n, h2); IO::st(io.h[2] + n, h3);
            if (c == 2 || c == mz - 3) {
                const int kh = c == 2 ? 1 : mz - 2, kz = c == 2 ? 0 : mz - 1;
                T hv[3][VX], zv[VX];
#pragma unroll
                for (int e = 0; e < VX; ++e) { hv[0][e] = T(0.5) * h1[e]; hv[1][e] = T(0.5) * h2[e]; hv[2][e] = T(0.5) * h3[e]; zv[e] = T(0); }
#pragma unroll
                for (int m = 0; m < 3; ++m) {
                    IO::st(io.h[m] + col + (long)kh * g.sz, hv[m]);
                    IO::st(io.h[m] + col + (long)kz * g.sz, zv);
                }
                // E0 on the wall rows is pointwise in the state there
#pragma unroll
                for (int kk = 0; kk < 2; ++kk) {
                    const int kw = kk == 0 ? kh : kz;
                    T f1[VX], f2[VX], f3[VX];
                    efield(col + (long)kw * g.sz, kw, f1, f2, f3);
                    IO::st(io.e[0] + col + (long)kw * g.sz, f1);
                    IO::st(io.e[1] + col + (long)kw * g.sz, f2);
                    IO::st(io.e[2] + col + (long)kw * g.sz, f3);
                }
            }
        }
#pragma unroll
        for (int s = 0; s < 4; ++s)
#pragma unroll
            for (int e = 0; e < VX; ++e) zq[s][e] = zq[s + 1][e];
    }
    cp_async_wait<0>();
}

}  // namespace dasha
