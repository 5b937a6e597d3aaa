// noalloc.cu -- dasha_current_noalloc: the smoothed current density J = S^4(curl(B - B0))
// computed without allocating any device memory.
//
// Who needs this: callers whose device memory is not theirs to allocate -- a host code that
// hands the GPU over to a memory manager owning every byte up front (a fixed pool sized at
// start-up, a cap enforced by a scheduler), code running where the CUDA allocator may not be
// called (inside a no-allocation phase of a larger application or while another component
// holds the allocator lock), and diagnostics that must not perturb a tight memory budget.
// dasha_current needs a context, whose buffers come from cudaMalloc; this entry point takes
// the caller's device input and output arrays and does its ping-pong passes in a fixed
// scratch array that is part of the library image.
//
// The scratch is a file-scope __device__ array of NOALLOC_SCRATCH_DOUBLES doubles (about 26 MB):
// every GPU that loads this library holds it until the process exits.  It holds one
// 3-field ping-pong buffer of at most NOALLOC_MAX_CELLS nodes and the 1-D stencil tables.
// All calls share it and it keeps the last call's contents; every byte a call reads is
// written earlier in the same call, so nothing has to be cleared.  Calls that overlap on the
// GPU (two streams, two host threads) race on it: serialise them.
#include "dasha_capi.h"
#include "mhd_kernels.cuh"
#include "coef.h"

#include <cmath>
#include <mutex>

using namespace dasha;

namespace {
constexpr long kMaxCells = DASHA_NOALLOC_MAX_CELLS;
constexpr int kAxisMax = DASHA_NOALLOC_MAX_AXIS;
constexpr int kTabPerAxis = 7;   // a1 b1 c1 d1 (first derivative), wp wm (difc), coordinate
constexpr long kTabDoubles = 3L * kTabPerAxis * kAxisMax;
constexpr long kScratchDoubles = 3 * kMaxCells + kTabDoubles;
static_assert(kScratchDoubles == DASHA_NOALLOC_SCRATCH_DOUBLES, "scratch size mismatch with dasha_capi.h");
constexpr int kMaxDevices = 64;

std::mutex g_mu;
double* g_dev_ptr[kMaxDevices] = {};   // device address of the scratch, per device ordinal
double g_host_tab[kTabDoubles];        // host staging of the tables (static: no heap use)
}  // namespace

static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

// One smoothing pass with the radial coefficient of avrgc (t3dsdsc.f:5981-5992) evaluated
// from the node coordinates, wall rows re-applied (bndryc t3dsdsc.f:2614-2642).
__global__ void k_noalloc_smooth(Geo<double> g, const double* xc, const double* yc, const double* zc,
                                 F3<double> in, F3<double> out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.mx) return;
    int jj = blockIdx.y, k = blockIdx.z;
    bool zero, half;
    int ks = wall_src(k, g.mz, zero, half);
    long c = (long)i + (long)jj * g.sy + (long)k * g.sz;
    if (zero) {
        out.f[0][c] = 0.0; out.f[1][c] = 0.0; out.f[2][c] = 0.0;
        return;
    }
    Nbr<double> n(g, i, jj, ks);
    double r = sqrt(xc[i] * xc[i] + yc[jj] * yc[jj] + zc[ks] * zc[ks]);
    double coef = 1.0 / 32.0 + (1.0 / 8.0 - 1.0 / 32.0) * 0.5 * (1 + tanh((r - 3.) / 3.));
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        double v = in.f[q][n.c] + coef * n.difc3(g, in.f[q]);
        out.f[q][c] = half ? 0.5 * v : v;
    }
}

// One-time set-up per device: the device address of the scratch array.  Host code must not
// use the symbol's name as an address (it is a host-side stand-in).
static int scratch_for_current_device(double** out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return DASHA_E_CUDA;
    if (!g_dev_ptr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) return DASHA_E_CUDA;
        g_dev_ptr[dev] = static_cast<double*>(p);
    }
    *out = g_dev_ptr[dev];
    return DASHA_OK;
}

extern "C" int dasha_current_noalloc(const dasha_grid_c* grid, const double* db_dev, double* cur_dev, void* stream) {
    if (!grid || !grid->x || !grid->y || !grid->z || !db_dev || !cur_dev) return DASHA_E_INVALID;
    const int mx = grid->mx, my = grid->my, mz = grid->mz;
    if (mx < 5 || my < 5 || mz < 7) return DASHA_E_INVALID;
    if (!(grid->periodic[0] == 1 && grid->periodic[1] == 1 && grid->periodic[2] == 0)) return DASHA_E_UNSUPPORTED;
    if ((long)mx * my * mz > kMaxCells || mx > kAxisMax || my > kAxisMax || mz > kAxisMax) return DASHA_E_NOSCRATCH;
    {   // the curl reads neighbours of B while it writes J: the two ranges must be disjoint
        const uintptr_t nb = 3u * sizeof(double) * (uintptr_t)mx * my * mz;
        const uintptr_t a = reinterpret_cast<uintptr_t>(db_dev), b = reinterpret_cast<uintptr_t>(cur_dev);
        if (a < b + nb && b < a + nb) return DASHA_E_INVALID;
    }
    const double* coords[3] = {grid->x, grid->y, grid->z};
    const int n[3] = {mx, my, mz};
    for (int d = 0; d < 3; ++d)
        for (int i = 0; i + 1 < n[d]; ++i)
            if (!(coords[d][i + 1] > coords[d][i])) return DASHA_E_INVALID;

    std::lock_guard<std::mutex> lock(g_mu);
    double* scratch = nullptr;
    if (int rc = scratch_for_current_device(&scratch)) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    // 1-D tables (host FP64), same construction as dasha_create
    for (int d = 0; d < 3; ++d) {
        const double* c = coords[d];
        const bool periodic = d < 2;
        const double L = periodic ? c[n[d] - 1] - c[0] + (c[1] - c[0]) : 0.0;
        auto at = [&](int i) {
            if (!periodic) return c[i];
            int q = 0;
            while (i < 0) { i += n[d]; --q; }
            while (i >= n[d]) { i -= n[d]; ++q; }
            return c[i] + q * L;
        };
        double* t = g_host_tab + (long)d * kTabPerAxis * kAxisMax;
        for (int q = 0; q < kTabPerAxis; ++q)
            for (int i = 0; i < n[d]; ++i) t[(long)q * kAxisMax + i] = 0.0;
        for (int i = 0; i < n[d]; ++i) {
            if (periodic || (i >= 2 && i <= n[d] - 3)) {
                double x0 = at(i), w1[4];
                if (!stencil_weights(at(i + 1) - x0, x0 - at(i - 1), at(i + 2) - x0, x0 - at(i - 2), 1, w1))
                    return DASHA_E_INVALID;
                for (int q = 0; q < 4; ++q) t[(long)q * kAxisMax + i] = w1[q];
            }
            if (periodic || (i >= 1 && i <= n[d] - 2)) {
                double xm = at(i - 1), x0 = at(i), xp = at(i + 1);
                t[4L * kAxisMax + i] = 2.0 * (xp - x0) / (xp - xm);
                t[5L * kAxisMax + i] = 2.0 * (x0 - xm) / (xp - xm);
            }
            t[6L * kAxisMax + i] = c[i];
        }
    }
    double* dtab = scratch + 3 * kMaxCells;
    if (cudaMemcpyAsync(dtab, g_host_tab, sizeof(double) * kTabDoubles, cudaMemcpyHostToDevice, st) != cudaSuccess)
        return DASHA_E_CUDA;

    Geo<double> g{};
    g.mx = mx; g.my = my; g.mz = mz; g.sy = mx; g.sz = (long)mx * my;
    const double* T[3];
    for (int d = 0; d < 3; ++d) T[d] = dtab + (long)d * kTabPerAxis * kAxisMax;
    g.a1x = T[0]; g.b1x = T[0] + kAxisMax; g.c1x = T[0] + 2 * kAxisMax; g.d1x = T[0] + 3 * kAxisMax;
    g.a1y = T[1]; g.b1y = T[1] + kAxisMax; g.c1y = T[1] + 2 * kAxisMax; g.d1y = T[1] + 3 * kAxisMax;
    g.a1z = T[2]; g.b1z = T[2] + kAxisMax; g.c1z = T[2] + 2 * kAxisMax; g.d1z = T[2] + 3 * kAxisMax;
    g.wpx = T[0] + 4 * kAxisMax; g.wmx = T[0] + 5 * kAxisMax;
    g.wpy = T[1] + 4 * kAxisMax; g.wmy = T[1] + 5 * kAxisMax;
    g.wpz = T[2] + 4 * kAxisMax; g.wmz = T[2] + 5 * kAxisMax;
    const double *xc = T[0] + 6 * kAxisMax, *yc = T[1] + 6 * kAxisMax, *zc = T[2] + 6 * kAxisMax;

    const long N = (long)mx * my * mz;
    F3<double> b, cur, tmp;
    for (int q = 0; q < 3; ++q) {
        b.f[q] = const_cast<double*>(db_dev) + q * N;
        cur.f[q] = cur_dev + q * N;
        tmp.f[q] = scratch + q * N;
    }
    dim3 blk(std::min(128, ((mx + 31) / 32) * 32));
    dim3 grd((mx + blk.x - 1) / blk.x, my, mz);
    // J1 = curl(B - B0) with the wall rows, then 4 passes cur -> scratch -> cur -> scratch -> cur
    k_curl<double><<<grd, blk, 0, st>>>(g, b, cur);
    for (int pass = 0; pass < 4; ++pass) {
        if (pass % 2 == 0) k_noalloc_smooth<<<grd, blk, 0, st>>>(g, xc, yc, zc, cur, tmp);
        else k_noalloc_smooth<<<grd, blk, 0, st>>>(g, xc, yc, zc, tmp, cur);
    }
    return cudaGetLastError() == cudaSuccess ? DASHA_OK : DASHA_E_CUDA;
}
