// k_zpv: one smoothing pass (avrg / avrgE / avrgc / avrgh / avrgtt, each with its bndry*),
// z-marching, register-blocked.
//
// A warp covers 32*VX consecutive x nodes (VX = 2 in FP32: each thread owns an aligned float2
// pair), a thread owns RY consecutive y rows of its pair, and the CTA marches up a chunk of z
// planes.  Every plane of the tile plus a 1-node x/y halo (no corners: the 7-point stencil has
// none) streams into an NS = D + 3 stage shared-memory ring with cp.async, D planes ahead.  The
// node's own values for planes c-1 and c stay in registers (z queue), so per plane a thread
// reads from shared memory only plane c+1 of its nodes, the x neighbours at the ends of its
// pair and the y neighbours above and below its strip: about 2 shared loads per node and field
// instead of 5.  Only planes c and c+1 are read in a plane step, so the stage refilled at step c
// (plane c+1+D, the stage of plane c-2) is neither of the two planes still read by threads in
// step c-1: one barrier per plane suffices; the first step also reads plane c-1 and so ends with
// a second barrier.  (Loading the planes by TMA instead, as ring-plane boxes with one mbarrier
// per stage, measured 7-40 % slower per pass on B200 in every arrangement tried: the passes are
// issue-bound and cp.async's per-thread copies cost about 2 % of their instructions.)
//
// TMA (k_zpv_tma; not built with -DDASHA_NO_TMA): a CTA whose ring box (x0-OFF .. x0+TX+OFF-1, rows
// y0-1 .. y0+TY) lies inside the grid loads each ring plane as NF `cp.async.bulk.tensor` boxes of
// exactly the ring plane's layout, issued by thread 0 against one mbarrier per stage; every thread
// waits (time-bounded) on the stages it reads before the plane's barrier.  CTAs whose halo wraps
// keep the cp.async copies.  The compute is the same code in both kernels; the engine picks one
// per launch.
//
// KINDS: 2 bits per output field, 0 radial coefficient, 1 constant 1/8, 2 x-profile cbx.
// MODE 0 writes the smoothed fields through the epilogue.  MODES 1 and 2 are the two passes of
// avrgtt on a compensated FP32 state (x, comp) whose value is x - comp: MODE 1 reads x in
// fields 0..NF/2-1 and comp in the rest and writes the first pass's increment d of x - comp;
// MODE 2 reads d and hands the two-pass increment 2 d + coef L(d) to a Kahan epilogue.
// Needs mx % 4 == 0 (16-byte row copies; a tile narrower than 32*VX at the x end is handled).
#pragma once

#include <type_traits>

#include "tma.cuh"

namespace dasha {

// the source fields of a pass as 3-D tensor maps with the box of one ring plane (k_zpv_tma)
struct ZpMaps { CUtensorMap m[8]; };

// VX consecutive values of a field, one access (8-byte aligned float pairs in FP32)
template <class T, int VX>
struct VIO;
template <class T>
struct VIO<T, 1> {
    static __device__ __forceinline__ void ld(const T* p, T (&v)[1]) { v[0] = *p; }
    static __device__ __forceinline__ void st(T* p, const T (&v)[1]) { *p = v[0]; }
};
template <>
struct VIO<float, 2> {
    static __device__ __forceinline__ void ld(const float* p, float (&v)[2]) {
        const float2 t = *reinterpret_cast<const float2*>(p);
        v[0] = t.x; v[1] = t.y;
    }
    static __device__ __forceinline__ void st(float* p, const float (&v)[2]) {
        *reinterpret_cast<float2*>(p) = make_float2(v[0], v[1]);
    }
};

// ---- epilogues: pre(i, p) loads the operands of the VX nodes starting at i (issued before
// the plane's barrier so that the loads overlap it), store(i, v, p) writes them; wall(i, v)
// writes a wall row (no prefetch) ----
template <class T, int NF, int VX>
struct VStore {
    T* f[NF];
    struct Pre {};
    __device__ __forceinline__ void pre(long, Pre&) const {}
    __device__ __forceinline__ void store(long i, const T (&v)[NF][VX], const Pre&) const { wall(i, v); }
    __device__ __forceinline__ void wall(long i, const T (&v)[NF][VX]) const {
#pragma unroll
        for (int q = 0; q < NF; ++q) VIO<T, VX>::st(f[q] + i, v[q]);
    }
};

template <class T, int NF, int VX>
struct VAcc {   // f = a + v  (a may alias f: each node is read and written by one thread)
    T* f[NF];
    const T* a[NF];
    struct Pre { T a[NF][VX]; };
    __device__ __forceinline__ void pre(long i, Pre& p) const {
#pragma unroll
        for (int q = 0; q < NF; ++q) VIO<T, VX>::ld(a[q] + i, p.a[q]);
    }
    __device__ __forceinline__ void store(long i, const T (&v)[NF][VX], const Pre& p) const {
#pragma unroll
        for (int q = 0; q < NF; ++q) {
            T w[VX];
#pragma unroll
            for (int x = 0; x < VX; ++x) w[x] = p.a[q][x] + v[q][x];
            VIO<T, VX>::st(f[q] + i, w);
        }
    }
    __device__ __forceinline__ void wall(long i, const T (&v)[NF][VX]) const {
        Pre p;
        pre(i, p);
        store(i, v, p);
    }
};

// f = v[q] + v[q + NO]: the pass over 2 NO fields writes the sums of the two halves (the last E
// smoothing pass and the fifth Hall pass, added into E, in one launch)
template <class T, int NO, int VX>
struct VSum {
    T* f[NO];
    struct Pre {};
    __device__ __forceinline__ void pre(long, Pre&) const {}
    __device__ __forceinline__ void store(long i, const T (&v)[2 * NO][VX], const Pre&) const { wall(i, v); }
    __device__ __forceinline__ void wall(long i, const T (&v)[2 * NO][VX]) const {
#pragma unroll
        for (int q = 0; q < NO; ++q) {
            T w[VX];
#pragma unroll
            for (int e = 0; e < VX; ++e) w[e] = v[q][e] + v[q + NO][e];
            VIO<T, VX>::st(f[q] + i, w);
        }
    }
};

// RK4 stage update with the smoothed xdif (stepon t3dsdsc.f:1090-1132): plain registers
// (base, acc = xm, x) in FP64; in FP32 acc holds only the increment and the base update of
// stage 4 is a Kahan step with the compensation comp (value = x - comp).
template <class T, int NF, int VX, bool KAHAN>
struct VRK {
    T* x[NF];
    const T* base[NF];
    T* acc[NF];
    T* comp[NF];
    int stage;
    double dt;
    struct Pre { T b[NF][VX], a[NF][VX], k[NF][VX]; };
    __device__ __forceinline__ void pre(long i, Pre& p) const {
#pragma unroll
        for (int q = 0; q < NF; ++q) {
#pragma unroll
            for (int e = 0; e < VX; ++e) { p.b[q][e] = T(0); p.a[q][e] = T(0); p.k[q][e] = T(0); }
            if (!(stage == 4 && !KAHAN)) VIO<T, VX>::ld(base[q] + i, p.b[q]);
            if (stage != 1) VIO<T, VX>::ld(acc[q] + i, p.a[q]);
            if (KAHAN && stage == 4) VIO<T, VX>::ld(comp[q] + i, p.k[q]);
        }
    }
    __device__ __forceinline__ void store(long i, const T (&v)[NF][VX], const Pre& p) const {
        const T tdt = T(dt);
#pragma unroll
        for (int q = 0; q < NF; ++q) {
            T xo[VX], ao[VX], ko[VX];
#pragma unroll
            for (int e = 0; e < VX; ++e) {
                const T kv = v[q][e], b = p.b[q][e];
                if (!KAHAN) {
                    if (stage == 1) { ao[e] = b + kv * tdt / T(6.); xo[e] = b + kv * tdt / T(2.); }
                    else if (stage == 2) { ao[e] = p.a[q][e] + kv * tdt / T(3.); xo[e] = b + kv * tdt / T(2.); }
                    else if (stage == 3) { ao[e] = p.a[q][e] + kv * tdt / T(3.); xo[e] = b + kv * tdt; }
                    else { xo[e] = p.a[q][e] + kv * tdt / T(6.); }
                } else {
                    if (stage == 1) { ao[e] = kv * tdt / T(6.); xo[e] = b + kv * tdt / T(2.); }
                    else if (stage == 2) { ao[e] = p.a[q][e] + kv * tdt / T(3.); xo[e] = b + kv * tdt / T(2.); }
                    else if (stage == 3) { ao[e] = p.a[q][e] + kv * tdt / T(3.); xo[e] = b + kv * tdt; }
                    else {
                        const T inc = p.a[q][e] + kv * tdt / T(6.);
                        const T y = inc - p.k[q][e];
                        const T t = b + y;
                        ko[e] = (t - b) - y;
                        xo[e] = t;
                    }
                }
            }
            VIO<T, VX>::st(x[q] + i, xo);
            if (stage < 4) VIO<T, VX>::st(acc[q] + i, ao);
            else if (KAHAN) VIO<T, VX>::st(comp[q] + i, ko);
        }
    }
    __device__ __forceinline__ void wall(long i, const T (&v)[NF][VX]) const {
        Pre p;
        pre(i, p);
        store(i, v, p);
    }
};

// MODE 2 epilogue: Kahan update of (x, comp) by the filter's increment, with the wall rows of
// the result set to the exact halves / zeros of rows 2 and mz-3 (bndrytt)
template <class T, int NF, int VX>
struct VKF {
    T* x[NF];
    T* comp[NF];
    struct Pre { T x[NF][VX], k[NF][VX]; };
    __device__ __forceinline__ void pre(long i, Pre& p) const {
#pragma unroll
        for (int q = 0; q < NF; ++q) { VIO<T, VX>::ld(x[q] + i, p.x[q]); VIO<T, VX>::ld(comp[q] + i, p.k[q]); }
    }
    __device__ __forceinline__ void store_rows(long i, bool wall, long ih, long iz, const T (&v)[NF][VX],
                                               const Pre& p) const {
#pragma unroll
        for (int q = 0; q < NF; ++q) {
            T t[VX], kk[VX], th[VX], kh[VX], z[VX];
#pragma unroll
            for (int e = 0; e < VX; ++e) {
                const T y = v[q][e] - p.k[q][e];
                t[e] = p.x[q][e] + y;
                kk[e] = (t[e] - p.x[q][e]) - y;
                th[e] = T(0.5) * t[e]; kh[e] = T(0.5) * kk[e]; z[e] = T(0);
            }
            VIO<T, VX>::st(x[q] + i, t);
            VIO<T, VX>::st(comp[q] + i, kk);
            if (wall) {
                VIO<T, VX>::st(x[q] + ih, th); VIO<T, VX>::st(comp[q] + ih, kh);
                VIO<T, VX>::st(x[q] + iz, z); VIO<T, VX>::st(comp[q] + iz, z);
            }
        }
    }
};

template <class T, int NF, int VX, int TYH, int RY, int D>
struct ZV {
    static constexpr int TX = 32 * VX;                // tile width (nodes)
    static constexpr int TY = TYH * RY;               // tile height
    static constexpr int EPC = 16 / (int)sizeof(T);   // elements per 16-byte copy
    static constexpr int OFF = EPC;                   // interior column offset in a ring row
    static constexpr int RS = TX + 2 * OFF;           // ring row stride
    static constexpr int NR = TY + 2;                 // rows y0-1 .. y0+TY
    static constexpr int SP = (RS * NR * (int)sizeof(T) + 127) / 128 * 128 / (int)sizeof(T);   // one field-plane, 128-byte aligned
    static constexpr int NS = D + 3;                  // ring stages
    static constexpr int CH = TX / EPC;               // 16-byte copies per full row
    static constexpr size_t smem() { return sizeof(T) * (size_t)NS * NF * SP; }
    // k_zpv_tma: the ring 128-byte aligned, then one mbarrier per stage
    static constexpr size_t smem_tma() { return 128 + smem() + 8 * NS; }
};

template <class T, int NF, unsigned KINDS, int VX, int TYH, int RY, int D, class Epi, int MODE, bool TMA>
__device__ __forceinline__ void zpv_body(const Geo<T>& g, const SrcFields<T, NF>& src, const Epi& epi, int chunk,
                                         const ZpMaps* maps) {
    using Z = ZV<T, NF, VX, TYH, RY, D>;
    constexpr int TX = Z::TX, TY = Z::TY, EPC = Z::EPC, OFF = Z::OFF, RS = Z::RS, SP = Z::SP, NS = Z::NS,
                  CH = Z::CH;
    constexpr int NT = 32 * TYH;
    constexpr int NO = MODE == 1 ? NF / 2 : NF;       // output fields
    static_assert(MODE != 1 || NF % 2 == 0, "MODE 1 reads (x, comp) field pairs");
    constexpr int NVEC = Z::NR * CH;                  // 16-byte copies per field-plane
    constexpr int NHAL = 2 * TY;                      // halo-column element copies
    using IO = VIO<T, VX>;
    extern __shared__ __align__(16) unsigned char zv_smem_raw[];
    unsigned char* sbase = zv_smem_raw;
    if constexpr (TMA) sbase += (128 - (smem_addr(zv_smem_raw) & 127)) & 127;
    T* ring = reinterpret_cast<T*>(sbase);            // [NS][NF][SP]
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const int wx = min(TX, g.mx - x0);
    const int mz = g.mz;
    const int k0 = blockIdx.z * chunk;
    const int k1 = min(k0 + chunk, mz);
    const int cA = max(k0, 2), cB = min(k1 - 1, mz - 3);
    if (cA > cB) return;
    // a CTA whose ring box lies inside the grid loads it by TMA (k_zpv_tma)
    const bool tma = TMA && x0 >= OFF && x0 + TX + OFF <= g.mx && y0 >= 1 && y0 + TY + 1 <= g.my;
    unsigned long long* bars = reinterpret_cast<unsigned long long*>(ring + (size_t)NS * NF * SP);
#ifndef DASHA_NO_TMA
    if constexpr (TMA) {
        if (tid == 0)
            for (int q = 0; q < NS; ++q) mbar_init(bars + q, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        __syncthreads();
    }
#else
    (void)bars;
    (void)maps;
#endif
    // this thread's copy slots (the same for every field and plane); -1 = none
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
                gsrc[q] = (long)(x0 + ch * EPC) + (long)pmod(y0 - 1 + r, g.my) * g.sy;
                sdst[q] = r * RS + OFF + ch * EPC;
            }
        } else if (sl < NVEC + NHAL) {
            const int h = sl - NVEC, r = h % TY + 1, side = h / TY;
            const int xx = side ? pmod(x0 + wx, g.mx) : pmod(x0 - 1, g.mx);
            gsrc[q] = (long)xx + (long)pmod(y0 - 1 + r, g.my) * g.sy;
            sdst[q] = r * RS + (side ? OFF + wx : OFF - 1);
        }
    }
    const int phi = cB + 1;
    auto issue = [&](int p) {
#ifndef DASHA_NO_TMA
        if (tma) {
            if (tid == 0 && p <= phi) {
                T* stg = ring + (long)(p % NS) * NF * SP;
                unsigned long long* bar = bars + p % NS;
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // after the stage's generic reads
                mbar_expect_tx(bar, (unsigned)(NF * RS * Z::NR * sizeof(T)));   // the boxes, not the padding
#pragma unroll
                for (int f = 0; f < NF; ++f) tma_load_3d(stg + f * SP, &maps->m[f], x0 - OFF, y0 - 1, p, bar);
            }
            return;
        }
#endif
        if (p <= phi) {
            T* stg = ring + (long)(p % NS) * NF * SP;
#pragma unroll
            for (int q = 0; q < NSL; ++q) {
                if (gsrc[q] >= 0) {
                    const long zo = gsrc[q] + (long)p * g.sz;
                    if (!DASHA_SPAN(zo, svec[q] ? EPC : 1, g.sz * (long)g.mz, BS_ZPV_LOAD)) continue;
#pragma unroll
                    for (int f = 0; f < NF; ++f) {
                        if (svec[q]) cp_async16(stg + f * SP + sdst[q], src.f[f] + zo);
                        else cp_async_elem(stg + f * SP + sdst[q], src.f[f] + zo);
                    }
                }
            }
        }
        cp_async_commit();
    };
#pragma unroll
    for (int p = 0; p < D + 2; ++p) issue(cA - 1 + p);   // planes cA-1 .. cA+D

    const int xl = VX * lane;                          // first own node in the tile
    const bool xon = xl < wx;
    const int gi = x0 + (xon ? xl : 0);
    T wpx[VX], wmx[VX], wsx[VX], cbx[VX], xx2[VX];
#pragma unroll
    for (int e = 0; e < VX; ++e) {
        wpx[e] = g.wpx[gi + e]; wmx[e] = g.wmx[gi + e]; cbx[e] = g.cbx[gi + e];
        wsx[e] = wpx[e] + wmx[e];
        xx2[e] = g.xc[gi + e] * g.xc[gi + e];
    }
    int gj[RY];
    T wpy[RY], wmy[RY], yy2[RY];
#pragma unroll
    for (int u = 0; u < RY; ++u) {
        gj[u] = y0 + w * RY + u;
        const int jj = gj[u] < g.my ? gj[u] : g.my - 1;
        wpy[u] = g.wpy[jj]; wmy[u] = g.wmy[jj];
        yy2[u] = g.yc[jj] * g.yc[jj];
    }
    T qm[RY][NF][VX], q0[RY][NF][VX];
    bool primed = false;
    for (int c = cA; c <= cB; ++c) {
        issue(c + 1 + D);
        const T wpz = g.wpz[c], wmz = g.wmz[c], wsz = wpz + wmz, zz2 = g.zc[c] * g.zc[c];
        typename Epi::Pre pre[RY];
#pragma unroll
        for (int u = 0; u < RY; ++u)
            if (xon && gj[u] < g.my && DASHA_SPAN((long)gi + (long)gj[u] * g.sy + (long)c * g.sz, VX, g.sz * (long)g.mz, BS_ZPV_STORE))
                epi.pre((long)gi + (long)gj[u] * g.sy + (long)c * g.sz, pre[u]);
#ifndef DASHA_NO_TMA
        if (tma) {
            // planes c-1 .. c+1 on the first step, then c+1
            bool late = false;
            for (int p = primed ? c + 1 : c - 1; p <= c + 1; ++p)
                if (!mbar_wait_bounded(bars + p % NS, (unsigned)(((p - (cA - 1)) / NS) & 1))) { late = true; break; }
            if (__syncthreads_or(late)) {
                // every box issued so far (planes up to c+1+D) lands before the CTA leaves
                if (tid == 0) atomicExch(&g_wait_timeout, 1u);
                for (int p = c - 1; p <= min(c + 1 + D, phi); ++p)
                    if (p >= cA - 1) mbar_wait_bounded(bars + p % NS, (unsigned)(((p - (cA - 1)) / NS) & 1));
                return;
            }
        } else
#endif
        {
            cp_async_wait<D>();
            __syncthreads();
        }
        const T* pc = ring + (long)(c % NS) * NF * SP;
        const T* pp = ring + (long)((c + 1) % NS) * NF * SP;
        const int base = (w * RY + 1) * RS + OFF + xl;   // ring index of row u = 0, own first node
        if (!primed) {
            const T* pm = ring + (long)((c + NS - 1) % NS) * NF * SP;
#pragma unroll
            for (int u = 0; u < RY; ++u)
#pragma unroll
                for (int f = 0; f < NF; ++f) {
                    IO::ld(pm + f * SP + base + u * RS, qm[u][f]);
                    IO::ld(pc + f * SP + base + u * RS, q0[u][f]);
                }
            primed = true;
            // plane c-1's stage is refilled at the next step: every thread must be done with it
            __syncthreads();
        }
        T qp[RY][NF][VX], ylo[NF][VX], yhi[NF][VX];
#pragma unroll
        for (int f = 0; f < NF; ++f) {
#pragma unroll
            for (int u = 0; u < RY; ++u) IO::ld(pp + f * SP + base + u * RS, qp[u][f]);
            IO::ld(pc + f * SP + base - RS, ylo[f]);
            IO::ld(pc + f * SP + base + RY * RS, yhi[f]);
        }
        const bool wall = c == 2 || c == mz - 3;
        const int kh = c == 2 ? 1 : mz - 2, kz = c == 2 ? 0 : mz - 1;
#pragma unroll
        for (int u = 0; u < RY; ++u) {
            if (!xon || gj[u] >= g.my) continue;
            T xle[NF], xri[NF];
#pragma unroll
            for (int f = 0; f < NF; ++f) {
                xle[f] = pc[f * SP + base + u * RS - 1];
                xri[f] = pc[f * SP + base + u * RS + VX];
            }
            T cr[VX];
#pragma unroll
            for (int e = 0; e < VX; ++e) cr[e] = any_kind0(KINDS, NO) ? radial_coef_fast(xx2[e] + yy2[u] + zz2) : T(0);
            // neighbour f, e in direction: x-, x+, y-, y+ (own strip from registers)
            auto nxm = [&](int f, int e) { return e > 0 ? q0[u][f][e > 0 ? e - 1 : 0] : xle[f]; };
            auto nxp = [&](int f, int e) { return e < VX - 1 ? q0[u][f][e < VX - 1 ? e + 1 : e] : xri[f]; };
            auto nym = [&](int f, int e) { return u > 0 ? q0[u > 0 ? u - 1 : 0][f][e] : ylo[f][e]; };
            auto nyp = [&](int f, int e) { return u < RY - 1 ? q0[u < RY - 1 ? u + 1 : u][f][e] : yhi[f][e]; };
            const long col = (long)gi + (long)gj[u] * g.sy;
            T val[NO][VX];
            if constexpr (MODE == 1) {
                // differences of x and of comp taken apart, then combined, so comp's bits are
                // not rounded away
#pragma unroll
                for (int f = 0; f < NO; ++f) {
                    const unsigned kind = (KINDS >> (2 * f)) & 3u;
#pragma unroll
                    for (int e = 0; e < VX; ++e) {
                        const T x0v = q0[u][f][e], k0v = q0[u][f + NO][e];
                        const T txp = (nxp(f, e) - x0v) - (nxp(f + NO, e) - k0v);
                        const T txm = (x0v - nxm(f, e)) - (k0v - nxm(f + NO, e));
                        const T typ = (nyp(f, e) - x0v) - (nyp(f + NO, e) - k0v);
                        const T tym = (x0v - nym(f, e)) - (k0v - nym(f + NO, e));
                        const T tzp = (qp[u][f][e] - x0v) - (qp[u][f + NO][e] - k0v);
                        const T tzm = (x0v - qm[u][f][e]) - (k0v - qm[u][f + NO][e]);
                        const T coef = kind == 0u ? cr[e] : (kind == 1u ? T(0.125) : cbx[e]);
                        val[f][e] = coef * (txp * wpx[e] - txm * wmx[e] + typ * wpy[u] - tym * wmy[u] + tzp * wpz - tzm * wmz);
                    }
                }
                if (DASHA_SPAN(col + (long)c * g.sz, VX, g.sz * (long)g.mz, BS_ZPV_STORE)) epi.store(col + (long)c * g.sz, val, pre[u]);
                if (wall && DASHA_SPAN(col + (long)kh * g.sz, VX, g.sz * (long)g.mz, BS_ZPV_WALL_LOAD) &&
                    DASHA_SPAN(col + (long)kz * g.sz, VX, g.sz * (long)g.mz, BS_ZPV_WALL_LOAD)) {
                    // wall rows of the pass result (row kh = half of row c, row kz = 0) as
                    // increments of x - comp
                    T hv[NO][VX], zv[NO][VX];
                    const long iz = col + (long)kz * g.sz;
#pragma unroll
                    for (int f = 0; f < NO; ++f) {
                        T xz[VX], kzv[VX];
                        IO::ld(src.f[f] + iz, xz);
                        IO::ld(src.f[f + NO] + iz, kzv);
#pragma unroll
                        for (int e = 0; e < VX; ++e) {
                            const T xw = c == 2 ? qm[u][f][e] : qp[u][f][e];
                            const T kw = c == 2 ? qm[u][f + NO][e] : qp[u][f + NO][e];
                            hv[f][e] = ((T(0.5) * q0[u][f][e] - xw) - (T(0.5) * q0[u][f + NO][e] - kw)) + T(0.5) * val[f][e];
                            zv[f][e] = kzv[e] - xz[e];
                        }
                    }
                    epi.wall(col + (long)kh * g.sz, hv);
                    epi.wall(iz, zv);
                }
            } else {
                // v0 + coef * sum_n w_n (f_n - v0) evaluated as (1 - coef W) v0 + coef sum_n w_n f_n,
                // W = sum_n w_n (about 6, coef W <= 0.75): 8 instructions per node and field
                // instead of 15, rounding still a few ulp of the field.  MODE 2: the two-pass
                // increment S(S(z)) - z = 2 d + coef L(d) from the first pass's increment d.
                T wsum[VX];
#pragma unroll
                for (int e = 0; e < VX; ++e) wsum[e] = wsx[e] + (wpy[u] + wmy[u]) + wsz;
                if constexpr (std::is_same<T, float>::value && VX == 2) {
                    // FP32 pairs: each operation on the thread's two nodes is one packed FFMA2 /
                    // FMUL2 (sm_100), with the roundings of the scalar form below
                    const float2 Wpx = make_float2(wpx[0], wpx[1]), Wmx = make_float2(wmx[0], wmx[1]);
                    const float2 Wpy = make_float2(wpy[u], wpy[u]), Wmy = make_float2(wmy[u], wmy[u]);
                    const float2 Wpz = make_float2(wpz, wpz), Wmz = make_float2(wmz, wmz);
                    const float2 Ws = make_float2(wsum[0], wsum[1]);
                    const float2 one = MODE == 2 ? make_float2(2.f, 2.f) : make_float2(1.f, 1.f);
#pragma unroll
                    for (int f = 0; f < NF; ++f) {
                        const unsigned kind = (KINDS >> (2 * f)) & 3u;
                        const float2 v0 = make_float2(q0[u][f][0], q0[u][f][1]);
                        float2 sn = __fmul2_rn(Wpx, make_float2(nxp(f, 0), nxp(f, 1)));
                        sn = __ffma2_rn(Wmx, make_float2(nxm(f, 0), nxm(f, 1)), sn);
                        sn = __ffma2_rn(Wpy, make_float2(nyp(f, 0), nyp(f, 1)), sn);
                        sn = __ffma2_rn(Wmy, make_float2(nym(f, 0), nym(f, 1)), sn);
                        sn = __ffma2_rn(Wpz, make_float2(qp[u][f][0], qp[u][f][1]), sn);
                        sn = __ffma2_rn(Wmz, make_float2(qm[u][f][0], qm[u][f][1]), sn);
                        const float2 cf = kind == 0u ? make_float2(cr[0], cr[1])
                                                     : (kind == 1u ? make_float2(0.125f, 0.125f) : make_float2(cbx[0], cbx[1]));
                        const float2 a = __ffma2_rn(make_float2(-cf.x, -cf.y), Ws, one);
                        const float2 r = __ffma2_rn(cf, sn, __fmul2_rn(a, v0));
                        val[f][0] = r.x;
                        val[f][1] = r.y;
                    }
                } else {
#pragma unroll
                    for (int f = 0; f < NF; ++f) {
                        const unsigned kind = (KINDS >> (2 * f)) & 3u;
#pragma unroll
                        for (int e = 0; e < VX; ++e) {
                            const T v0 = q0[u][f][e];
                            T sn = wpx[e] * nxp(f, e);
                            sn = fma(wmx[e], nxm(f, e), sn);
                            sn = fma(wpy[u], nyp(f, e), sn);
                            sn = fma(wmy[u], nym(f, e), sn);
                            sn = fma(wpz, qp[u][f][e], sn);
                            sn = fma(wmz, qm[u][f][e], sn);
                            const T coef = kind == 0u ? cr[e] : (kind == 1u ? T(0.125) : cbx[e]);
                            const T a = fma(-coef, wsum[e], MODE == 2 ? T(2) : T(1));
                            val[f][e] = fma(coef, sn, a * v0);
                        }
                    }
                }
                if constexpr (MODE == 2) {
                    if (DASHA_SPAN(col + (long)c * g.sz, VX, g.sz * (long)g.mz, BS_ZPV_STORE) &&
                        (!wall || (DASHA_SPAN(col + (long)kh * g.sz, VX, g.sz * (long)g.mz, BS_ZPV_STORE) &&
                                   DASHA_SPAN(col + (long)kz * g.sz, VX, g.sz * (long)g.mz, BS_ZPV_STORE))))
                        epi.store_rows(col + (long)c * g.sz, wall, col + (long)kh * g.sz, col + (long)kz * g.sz, val, pre[u]);
                } else {
                    if (DASHA_SPAN(col + (long)c * g.sz, VX, g.sz * (long)g.mz, BS_ZPV_STORE)) epi.store(col + (long)c * g.sz, val, pre[u]);
                    if (wall && DASHA_SPAN(col + (long)kh * g.sz, VX, g.sz * (long)g.mz, BS_ZPV_STORE) &&
                        DASHA_SPAN(col + (long)kz * g.sz, VX, g.sz * (long)g.mz, BS_ZPV_STORE)) {
                        T hv[NF][VX], zv[NF][VX];
#pragma unroll
                        for (int f = 0; f < NF; ++f)
#pragma unroll
                            for (int e = 0; e < VX; ++e) { hv[f][e] = T(0.5) * val[f][e]; zv[f][e] = T(0); }
                        epi.wall(col + (long)kh * g.sz, hv);
                        epi.wall(col + (long)kz * g.sz, zv);
                    }
                }
            }
        }
#pragma unroll
        for (int u = 0; u < RY; ++u)
#pragma unroll
            for (int f = 0; f < NF; ++f)
#pragma unroll
                for (int e = 0; e < VX; ++e) { qm[u][f][e] = q0[u][f][e]; q0[u][f][e] = qp[u][f][e]; }
    }
    cp_async_wait<0>();
    if constexpr (has_finish<Epi>::value) epi.finish();   // the fused CFL maximum (WithCfl)
}

template <class T, int NF, unsigned KINDS, int VX, int TYH, int RY, int D, class Epi, int MODE = 0>
__global__ void __launch_bounds__(32 * TYH) k_zpv(Geo<T> g, SrcFields<T, NF> src, Epi epi, int chunk) {
    zpv_body<T, NF, KINDS, VX, TYH, RY, D, Epi, MODE, false>(g, src, epi, chunk, nullptr);
}

#ifndef DASHA_NO_TMA
template <class T, int NF, unsigned KINDS, int VX, int TYH, int RY, int D, class Epi, int MODE = 0>
__global__ void __launch_bounds__(32 * TYH) k_zpv_tma(Geo<T> g, SrcFields<T, NF> src, Epi epi, int chunk,
                                                      const __grid_constant__ ZpMaps maps) {
    zpv_body<T, NF, KINDS, VX, TYH, RY, D, Epi, MODE, true>(g, src, epi, chunk, &maps);
}
#endif

}  // namespace dasha
