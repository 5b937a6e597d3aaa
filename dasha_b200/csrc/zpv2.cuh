// k_zpv2: two consecutive smoothing passes of the same kind in one z-march (temporal
// blocking), so the fields between the passes never go to HBM.
//
// A warp covers 32*VX consecutive x nodes (VX = 2 in FP32: float pairs), one row per warp.
// Warps 1..TY own the tile rows y0..y0+TY-1; warps 0 and TY+1 own the halo rows y0-1 and
// y0+TY, whose first-pass values the second pass needs as y neighbours.  Per plane step p:
//   - the input plane p+1+D is issued into an NS = D+4 stage ring (16-byte cp.async rows plus
//     the x-halo columns x0-2, x0-1, x0+wx, x0+wx+1, rows y0-2 .. y0+TY+1);
//   - one barrier: input plane p+1 has landed, and every thread's first-pass plane p-1 is
//     written;
//   - the first pass at plane p (level 1) for the own nodes (z neighbours from a register
//     queue), and, by the end lanes of the tile rows, for the x-halo columns x0-1 and x0+wx
//     (z neighbours from the ring, which keeps planes p-1 .. p+1); level 1 goes to a 3-plane
//     shared ring and the own values also to a register queue of planes p-2 .. p;
//   - the second pass at plane p-1 for the tile rows: z neighbours from the level-1 register
//     queue, x and y neighbours from level-1 plane p-1 in shared memory; result to the
//     epilogue.
// Level-1 plane p is written at step p into stage p % 3 and read at step p+1; stage p % 3
// held plane p-3, last read at step p-2, and every thread passed step p-1's barrier after it:
// no second barrier.  The input stage refilled at step p (plane p+1+D) held plane p-3, last
// read at step p-2: NS = D + 4.  The wall rows follow bndry after each pass: level-1 rows 1
// and mz-2 are half of rows 2 and mz-3 (own register queue; no x/y neighbour needs them) and
// the result's wall rows are written with the result.
//
// KINDS: 2 bits per field, 0 radial coefficient, 1 constant 1/8, 2 x-profile cbx; the same
// kind for both passes.  Needs mx % 4 == 0 (16-byte row copies; a narrower last x tile is handled).
#pragma once

#include <type_traits>

namespace dasha {

template <class T, int NF, int VX, int TY, int D>
struct ZV2 {
    static constexpr int TX = 32 * VX;                // tile width
    static constexpr int NW = TY + 2;                 // warps: halo row, TY tile rows, halo row
    static constexpr int EPC = 16 / (int)sizeof(T);   // elements per 16-byte copy
    static constexpr int OFF = EPC;                   // interior column offset in a ring row (>= 2)
    static constexpr int RS = TX + 2 * OFF;           // row stride of both rings
    static constexpr int NRI = TY + 4;                // input rows y0-2 .. y0+TY+1
    static constexpr int SPI = NRI * RS;              // one input field-plane
    static constexpr int NSI = D + 4;                 // input stages
    static constexpr int NR1 = TY + 2;                // level-1 rows y0-1 .. y0+TY
    static constexpr int SP1 = NR1 * RS;              // one level-1 field-plane
    static constexpr int CH = TX / EPC;               // 16-byte copies per full row
    static constexpr size_t smem() { return sizeof(T) * ((size_t)NSI * NF * SPI + 3 * (size_t)NF * SP1); }
};

template <class T, int NF, unsigned KINDS, int VX, int TY, int D, class Epi>
__global__ void __launch_bounds__(32 * (TY + 2)) k_zpv2(Geo<T> g, SrcFields<T, NF> src, Epi epi, int chunk) {
    using Z = ZV2<T, NF, VX, TY, D>;
    constexpr int TX = Z::TX, EPC = Z::EPC, OFF = Z::OFF, RS = Z::RS, NRI = Z::NRI, SPI = Z::SPI, NSI = Z::NSI,
                  SP1 = Z::SP1, CH = Z::CH;
    constexpr int NT = 32 * Z::NW;
    constexpr int NVEC = NRI * CH;                    // 16-byte copies per field-plane
    constexpr int NHAL = 4 * NRI;                     // halo-column element copies per field-plane
    using IO = VIO<T, VX>;
    extern __shared__ __align__(16) unsigned char zv2_smem_raw[];
    T* ring = reinterpret_cast<T*>(zv2_smem_raw);     // [NSI][NF][SPI]
    T* lv1 = ring + (size_t)NSI * NF * SPI;           // [3][NF][SP1]
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const int wx = min(TX, g.mx - x0);
    const int mz = g.mz;
    const int k0 = blockIdx.z * chunk;
    const int k1 = min(k0 + chunk, mz);
    const int oA = max(k0, 2), oB = min(k1 - 1, mz - 3);   // output planes of this CTA
    if (oA > oB) return;
    const int pA = max(oA - 1, 2), pB = min(oB + 1, mz - 3);   // level-1 planes
    // copy slots of this thread (the same for every field and plane); -1 = none
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
            const int h = sl - NVEC, r = h % NRI, side = h / NRI;   // side 0..3: x0-2, x0-1, x0+wx, x0+wx+1
            const int dx = side < 2 ? side - 2 : wx + side - 2;
            gsrc[q] = (long)pmod(x0 + dx, g.mx) + (long)pmod(y0 - 2 + r, g.my) * g.sy;
            sdst[q] = r * RS + OFF + dx;
        }
    }
    const int phi = pB + 1;                           // last input plane
    auto issue = [&](int p) {
        if (p <= phi) {
            T* stg = ring + (size_t)(p % NSI) * NF * SPI;
#pragma unroll
            for (int q = 0; q < NSL; ++q) {
                if (gsrc[q] >= 0) {
                    const long zo = gsrc[q] + (long)p * g.sz;
                    if (!DASHA_SPAN(zo, svec[q] ? EPC : 1, g.sz * (long)g.mz, BS_ZPV2_LOAD)) continue;
#pragma unroll
                    for (int f = 0; f < NF; ++f) {
                        if (svec[q]) cp_async16(stg + f * SPI + sdst[q], src.f[f] + zo);
                        else cp_async_elem(stg + f * SPI + sdst[q], src.f[f] + zo);
                    }
                }
            }
        }
        cp_async_commit();
    };
#pragma unroll
    for (int p = 0; p < D + 2; ++p) issue(pA - 1 + p);   // input planes pA-1 .. pA+D

    // this warp's row: rr = -1 .. TY (ring row rr+2 in the input, rr+1 in level 1)
    const int rr = w - 1;
    const bool trow = rr >= 0 && rr < TY;             // a tile row (second pass here)
    const int gy = pmod(y0 + rr, g.my);               // level 1 of a row beyond my is the wrapped row's
    const bool yon = y0 + rr < g.my;                  // (the y neighbour of row my-1); no output there
    const int xl = VX * lane;
    const bool xon = xl < wx;
    const int gi = x0 + (xon ? xl : 0);
    const int lastl = wx / VX - 1;                    // last active lane
    // extra level-1 node of the end lanes on tile rows: x0-1 (lane 0), x0+wx (last lane)
    const bool xtra = trow && (lane == 0 || lane == lastl);
    const int xe = lane == 0 ? -1 : wx;               // its column relative to x0
    const int gxe = pmod(x0 + xe, g.mx);
    T wpx[VX], wmx[VX], wsx[VX], cbx[VX], xx2[VX];
#pragma unroll
    for (int e = 0; e < VX; ++e) {
        wpx[e] = g.wpx[gi + e]; wmx[e] = g.wmx[gi + e]; cbx[e] = g.cbx[gi + e];
        wsx[e] = wpx[e] + wmx[e];
        xx2[e] = g.xc[gi + e] * g.xc[gi + e];
    }
    const T wpy = g.wpy[gy], wmy = g.wmy[gy], yy2 = g.yc[gy] * g.yc[gy];
    const T ewpx = g.wpx[gxe], ewmx = g.wmx[gxe], ecbx = g.cbx[gxe], exx2 = g.xc[gxe] * g.xc[gxe];
    // coefficient of field f at a node with squared radius part r2 (= x^2 + y^2) and plane zz2
    auto coef_of = [&](int f, T cb, T r2, T zz2) -> T {
        const unsigned kind = (KINDS >> (2 * f)) & 3u;
        return kind == 0u ? radial_coef_fast(r2 + zz2) : (kind == 1u ? T(0.125) : cb);
    };

    const int ri = rr + 2;                            // input ring row
    const int r1 = rr + 1;                            // level-1 ring row
    T qm[NF][VX], q0[NF][VX];                         // input planes p-1, p (own nodes)
    T la[NF][VX], lb[NF][VX], lc[NF][VX];             // level 1, planes p-2, p-1, p (own nodes)
    bool primed = false;
    for (int p = pA; p <= pB; ++p) {
        issue(p + 1 + D);
        const int q = p - 1;                          // second-pass plane of this step
        const bool out = trow && yon && xon && q >= oA && q <= oB;
        typename Epi::Pre pre;
        if (out && DASHA_SPAN((long)gi + (long)gy * g.sy + (long)q * g.sz, VX, g.sz * (long)g.mz, BS_ZPV2_STORE))
            epi.pre((long)gi + (long)gy * g.sy + (long)q * g.sz, pre);
        cp_async_wait<D>();
        __syncthreads();
        const T* pm = ring + (size_t)((p + NSI - 1) % NSI) * NF * SPI;
        const T* pc = ring + (size_t)(p % NSI) * NF * SPI;
        const T* pp = ring + (size_t)((p + 1) % NSI) * NF * SPI;
        const int me = ri * RS + OFF + xl;
        if (!primed) {
#pragma unroll
            for (int f = 0; f < NF; ++f) {
                IO::ld(pm + f * SPI + me, qm[f]);
                IO::ld(pc + f * SPI + me, q0[f]);
            }
        }
        T qp[NF][VX];
#pragma unroll
        for (int f = 0; f < NF; ++f) IO::ld(pp + f * SPI + me, qp[f]);
        // ---- level 1 at plane p ----
        const T wpz = g.wpz[p], wmz = g.wmz[p], wsz = wpz + wmz, zz2 = g.zc[p] * g.zc[p];
        T* l1p = lv1 + (size_t)(p % 3) * NF * SP1;
        T l1[NF][VX];
        if (xon) {
            T ylo[NF][VX], yhi[NF][VX], xle[NF], xri[NF];
#pragma unroll
            for (int f = 0; f < NF; ++f) {
                IO::ld(pc + f * SPI + me - RS, ylo[f]);
                IO::ld(pc + f * SPI + me + RS, yhi[f]);
                xle[f] = pc[f * SPI + me - 1];
                xri[f] = pc[f * SPI + me + VX];
            }
            if constexpr (std::is_same<T, float>::value && VX == 2) {
                // FP32 pairs as packed FFMA2 / FMUL2, with the roundings of the scalar form below
                const float2 Wpx = make_float2(wpx[0], wpx[1]), Wmx = make_float2(wmx[0], wmx[1]);
                const float2 Wpy = make_float2(wpy, wpy), Wmy = make_float2(wmy, wmy);
                const float2 Wpz = make_float2(wpz, wpz), Wmz = make_float2(wmz, wmz);
                const float2 Ws = make_float2(wsx[0] + (wpy + wmy) + wsz, wsx[1] + (wpy + wmy) + wsz);
#pragma unroll
                for (int f = 0; f < NF; ++f) {
                    float2 sn = __fmul2_rn(Wpx, make_float2(q0[f][1], xri[f]));
                    sn = __ffma2_rn(Wmx, make_float2(xle[f], q0[f][0]), sn);
                    sn = __ffma2_rn(Wpy, make_float2(yhi[f][0], yhi[f][1]), sn);
                    sn = __ffma2_rn(Wmy, make_float2(ylo[f][0], ylo[f][1]), sn);
                    sn = __ffma2_rn(Wpz, make_float2(qp[f][0], qp[f][1]), sn);
                    sn = __ffma2_rn(Wmz, make_float2(qm[f][0], qm[f][1]), sn);
                    const float2 cf = make_float2(coef_of(f, cbx[0], xx2[0] + yy2, zz2), coef_of(f, cbx[1], xx2[1] + yy2, zz2));
                    const float2 a = __ffma2_rn(make_float2(-cf.x, -cf.y), Ws, make_float2(1.f, 1.f));
                    const float2 r = __ffma2_rn(cf, sn, __fmul2_rn(a, make_float2(q0[f][0], q0[f][1])));
                    l1[f][0] = r.x;
                    l1[f][1] = r.y;
                }
            } else {
#pragma unroll
                for (int f = 0; f < NF; ++f)
#pragma unroll
                    for (int e = 0; e < VX; ++e) {
                        const T v0 = q0[f][e];
                        T sn = wpx[e] * (e < VX - 1 ? q0[f][e < VX - 1 ? e + 1 : e] : xri[f]);
                        sn = fma(wmx[e], e > 0 ? q0[f][e > 0 ? e - 1 : 0] : xle[f], sn);
                        sn = fma(wpy, yhi[f][e], sn);
                        sn = fma(wmy, ylo[f][e], sn);
                        sn = fma(wpz, qp[f][e], sn);
                        sn = fma(wmz, qm[f][e], sn);
                        const T c = coef_of(f, cbx[e], xx2[e] + yy2, zz2);
                        const T a = fma(-c, wsx[e] + (wpy + wmy) + wsz, T(1));
                        l1[f][e] = fma(c, sn, a * v0);
                    }
            }
#pragma unroll
            for (int f = 0; f < NF; ++f) IO::st(l1p + f * SP1 + r1 * RS + OFF + xl, l1[f]);
        }
        if (xtra) {   // the level-1 x-halo node of this tile row
            const int ie = ri * RS + OFF + xe;
#pragma unroll
            for (int f = 0; f < NF; ++f) {
                const T* a0 = pc + f * SPI;
                const T v0 = a0[ie];
                T sn = ewpx * a0[ie + 1];
                sn = fma(ewmx, a0[ie - 1], sn);
                sn = fma(wpy, a0[ie + RS], sn);
                sn = fma(wmy, a0[ie - RS], sn);
                sn = fma(wpz, pp[f * SPI + ie], sn);
                sn = fma(wmz, pm[f * SPI + ie], sn);
                const T c = coef_of(f, ecbx, exx2 + yy2, zz2);
                const T a = fma(-c, (ewpx + ewmx) + (wpy + wmy) + wsz, T(1));
                l1p[f * SP1 + r1 * RS + OFF + xe] = fma(c, sn, a * v0);
            }
        }
        // level-1 register queue: planes p-2, p-1, p; below plane 2 the wall row (half of row 2)
#pragma unroll
        for (int f = 0; f < NF; ++f)
#pragma unroll
            for (int e = 0; e < VX; ++e) {
                if (!primed) {
                    la[f][e] = T(0);
                    lb[f][e] = T(0.5) * l1[f][e];   // plane 1 when p == 2 (used only then)
                } else {
                    la[f][e] = lb[f][e];
                    lb[f][e] = lc[f][e];
                }
                lc[f][e] = l1[f][e];
            }
        primed = true;
        // ---- second pass at plane q = p-1 (level-1 plane q written at step q, before this
        // step's barrier) ----
        if (out) {
            const T* l1q = lv1 + (size_t)(q % 3) * NF * SP1;
            const int m1 = r1 * RS + OFF + xl;
            const T zwp = g.wpz[q], zwm = g.wmz[q], zws = zwp + zwm, qz2 = g.zc[q] * g.zc[q];
            T val[NF][VX];
#pragma unroll
            for (int f = 0; f < NF; ++f) {
                T ylo[VX], yhi[VX];
                IO::ld(l1q + f * SP1 + m1 - RS, ylo);
                IO::ld(l1q + f * SP1 + m1 + RS, yhi);
                const T xle = l1q[f * SP1 + m1 - 1], xri = l1q[f * SP1 + m1 + VX];
                if constexpr (std::is_same<T, float>::value && VX == 2) {
                    float2 sn = __fmul2_rn(make_float2(wpx[0], wpx[1]), make_float2(lb[f][1], xri));
                    sn = __ffma2_rn(make_float2(wmx[0], wmx[1]), make_float2(xle, lb[f][0]), sn);
                    sn = __ffma2_rn(make_float2(wpy, wpy), make_float2(yhi[0], yhi[1]), sn);
                    sn = __ffma2_rn(make_float2(wmy, wmy), make_float2(ylo[0], ylo[1]), sn);
                    sn = __ffma2_rn(make_float2(zwp, zwp), make_float2(lc[f][0], lc[f][1]), sn);
                    sn = __ffma2_rn(make_float2(zwm, zwm), make_float2(la[f][0], la[f][1]), sn);
                    const float2 cf = make_float2(coef_of(f, cbx[0], xx2[0] + yy2, qz2), coef_of(f, cbx[1], xx2[1] + yy2, qz2));
                    const float2 ws = make_float2(wsx[0] + (wpy + wmy) + zws, wsx[1] + (wpy + wmy) + zws);
                    const float2 a = __ffma2_rn(make_float2(-cf.x, -cf.y), ws, make_float2(1.f, 1.f));
                    const float2 r = __ffma2_rn(cf, sn, __fmul2_rn(a, make_float2(lb[f][0], lb[f][1])));
                    val[f][0] = r.x;
                    val[f][1] = r.y;
                } else {
#pragma unroll
                    for (int e = 0; e < VX; ++e) {
                        const T v0 = lb[f][e];
                        T sn = wpx[e] * (e < VX - 1 ? lb[f][e < VX - 1 ? e + 1 : e] : xri);
                        sn = fma(wmx[e], e > 0 ? lb[f][e > 0 ? e - 1 : 0] : xle, sn);
                        sn = fma(wpy, yhi[e], sn);
                        sn = fma(wmy, ylo[e], sn);
                        sn = fma(zwp, lc[f][e], sn);
                        sn = fma(zwm, la[f][e], sn);
                        const T c = coef_of(f, cbx[e], xx2[e] + yy2, qz2);
                        const T a = fma(-c, wsx[e] + (wpy + wmy) + zws, T(1));
                        val[f][e] = fma(c, sn, a * v0);
                    }
                }
            }
            const long col = (long)gi + (long)gy * g.sy;
            if (DASHA_SPAN(col + (long)q * g.sz, VX, g.sz * (long)g.mz, BS_ZPV2_STORE)) epi.store(col + (long)q * g.sz, val, pre);
            if (q == 2) {
                T hv[NF][VX], zv[NF][VX];
#pragma unroll
                for (int f = 0; f < NF; ++f)
#pragma unroll
                    for (int e = 0; e < VX; ++e) { hv[f][e] = T(0.5) * val[f][e]; zv[f][e] = T(0); }
                epi.wall(col + 1L * g.sz, hv);
                epi.wall(col, zv);
            }
        }
#pragma unroll
        for (int f = 0; f < NF; ++f)
#pragma unroll
            for (int e = 0; e < VX; ++e) { qm[f][e] = q0[f][e]; q0[f][e] = qp[f][e]; }
    }
    // last output plane mz-3: its level-1 plane above is the wall row mz-2 = half of mz-3
    if (oB == mz - 3) {
        __syncthreads();   // level-1 plane mz-3 of every thread
        const int q = oB;
        if (trow && yon && xon) {
            typename Epi::Pre pre;
            const long col = (long)gi + (long)gy * g.sy;
            if (DASHA_SPAN(col + (long)q * g.sz, VX, g.sz * (long)g.mz, BS_ZPV2_STORE)) epi.pre(col + (long)q * g.sz, pre);
            const T* l1q = lv1 + (size_t)(q % 3) * NF * SP1;
            const int m1 = r1 * RS + OFF + xl;
            const T zwp = g.wpz[q], zwm = g.wmz[q], zws = zwp + zwm, qz2 = g.zc[q] * g.zc[q];
            T val[NF][VX];
#pragma unroll
            for (int f = 0; f < NF; ++f) {
                T ylo[VX], yhi[VX];
                IO::ld(l1q + f * SP1 + m1 - RS, ylo);
                IO::ld(l1q + f * SP1 + m1 + RS, yhi);
                const T xle = l1q[f * SP1 + m1 - 1], xri = l1q[f * SP1 + m1 + VX];
#pragma unroll
                for (int e = 0; e < VX; ++e) {
                    const T v0 = lc[f][e];            // plane mz-3
                    T sn = wpx[e] * (e < VX - 1 ? lc[f][e < VX - 1 ? e + 1 : e] : xri);
                    sn = fma(wmx[e], e > 0 ? lc[f][e > 0 ? e - 1 : 0] : xle, sn);
                    sn = fma(wpy, yhi[e], sn);
                    sn = fma(wmy, ylo[e], sn);
                    sn = fma(zwp, T(0.5) * lc[f][e], sn);   // plane mz-2: wall row of level 1
                    sn = fma(zwm, lb[f][e], sn);            // plane mz-4
                    const T c = coef_of(f, cbx[e], xx2[e] + yy2, qz2);
                    const T a = fma(-c, wsx[e] + (wpy + wmy) + zws, T(1));
                    val[f][e] = fma(c, sn, a * v0);
                }
            }
            if (DASHA_SPAN(col + (long)q * g.sz, VX, g.sz * (long)g.mz, BS_ZPV2_STORE)) epi.store(col + (long)q * g.sz, val, pre);
            T hv[NF][VX], zv[NF][VX];
#pragma unroll
            for (int f = 0; f < NF; ++f)
#pragma unroll
                for (int e = 0; e < VX; ++e) { hv[f][e] = T(0.5) * val[f][e]; zv[f][e] = T(0); }
            epi.wall(col + (long)(mz - 2) * g.sz, hv);
            epi.wall(col + (long)(mz - 1) * g.sz, zv);
        }
    }
    cp_async_wait<0>();
}

}  // namespace dasha
