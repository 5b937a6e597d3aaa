// dasha_capi.cu -- host side of libdasha.so: context, device buffers, coefficient set-up and
// the C-ABI declared in include/dasha_capi.h.  All device work is in mhd_kernels.cuh.
#include "dasha_capi.h"
#include "mhd_kernels.cuh"
#include "engine.cuh"
#include "fortran_format.h"
#include "fortran_records.h"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>
#include <new>

using namespace dasha;

#include "coef.h"

struct Axis {
    int n;
    bool periodic;
    std::vector<double> c;    // coordinates
    double L = 0;             // period
    double at(int i) const {  // coordinate continued across the wrap
        if (!periodic) return c[i];
        int q = 0;
        while (i < 0) { i += n; --q; }
        while (i >= n) { i -= n; ++q; }
        return c[i] + q * L;
    }
};

namespace dasha {
template <class T>
static EngineBase* make_engine(int mx, int my, int mz, const dasha_params_c& p, cudaStream_t st,
                               const HostTables& H, Status& s) {
    Engine<T>* e = new Engine<T>();
    s = e->init(mx, my, mz, p, st, H);
    return e;
}
EngineBase* make_engine_f64(int mx, int my, int mz, const dasha_params_c& p, cudaStream_t st, const HostTables& H,
                            Status& s) {
    return make_engine<double>(mx, my, mz, p, st, H, s);
}
EngineBase* make_engine_f32(int mx, int my, int mz, const dasha_params_c& p, cudaStream_t st, const HostTables& H,
                            Status& s) {
    return make_engine<float>(mx, my, mz, p, st, H, s);
}
}  // namespace dasha

// ---------------------------------------------------------------------------------------
struct dasha_ctx {
    int mx = 0, my = 0, mz = 0;
    long N = 0;
    dasha_params_c P{};
    int device = 0;
    cudaStream_t st = nullptr;
    std::string err;
    int sticky = 0;
    Axis ax, ay, az;
    EngineBase* eng = nullptr;
    bool eq_set = false, state_set = false;
    bool bounded = false;     // periodic = {0,0,0}: the reference's bounded configuration
    double dt0 = 0.;
    bool have_dt0 = false;
    // z-slab contexts (dasha_create_slab): slab `slab` of `nslabs`, own global rows zfirst ..,
    // local planes = global rows zfirst-2 .. zfirst+mz-3, global grid mzg planes
    int nslabs = 1, slab = 0, zfirst = 2, mzg = 0;
    std::unique_ptr<Halo> halo;
    std::shared_ptr<LocalGroup> group;   // the in-process group it was linked into
    bool is_slab() const { return nslabs > 1; }
};

static int fail(dasha_ctx* c, int code, const std::string& msg) {
    if (c) {
        c->err = msg;
        if (code == DASHA_E_CUDA) c->sticky = code;
    }
    return code;
}

#define CAPI_GUARD(ctx)                                                                       \
    if (!(ctx)) return DASHA_E_INVALID;                                                       \
    if ((ctx)->sticky) return (ctx)->sticky;

// entry points over the whole grid (outputs, restart, adjoint) that a z-slab context refuses
#define SLAB_UNSUPPORTED(c, what)                                                              \
    if ((c)->is_slab()) return fail((c), DASHA_E_UNSUPPORTED, what " needs the whole grid: not on a z-slab context");

// a z-slab's own setdt / stepon / current: a slab of a one-process-per-GPU run (dasha_slab_nccl);
// the slabs of one process step together through the dasha_group_* calls
static int slab_single_call(dasha_ctx* c) {
    if (!c->is_slab()) return DASHA_OK;
    if (!c->halo) return fail(c, DASHA_E_STATE, "z-slab not joined to its neighbours (dasha_slab_link or dasha_slab_nccl)");
    if (!c->halo->per_process())
        return fail(c, DASHA_E_STATE, "linked slabs step together: dasha_group_setdt / dasha_group_stepon / dasha_group_current");
    return DASHA_OK;
}

static int from_status(dasha_ctx* c, const Status& s) {
    if (s.code == DASHA_OK) return DASHA_OK;
    return fail(c, s.code, s.msg);
}

// Runs the body of an entry point: a host exception (allocation, thread start) becomes a
// status, as no exception may cross the C-ABI.
#ifdef DASHA_BOUNDS
// the checking build: after every entry point, the first out-of-range access its kernels met
static int bounds_status(dasha_ctx* c, int rc) {
    static const char* names[BS_COUNT] = {"k_zpv ring load", "k_zpv node", "k_zpv wall row", "k_zpv2 ring load",
                                          "k_zpv2 node", "k_zcurl ring load", "k_zcurl store", "k_zhydro ring load",
                                          "k_zhydro node load", "k_zhydro store", "k_zeh ring load",
                                          "k_zeh node load", "k_zeh store"};
    if (!c || !c->st) return rc;
    unsigned long long hit = 0;
    if (cudaStreamSynchronize(c->st) != cudaSuccess ||
        cudaMemcpyFromSymbol(&hit, g_bounds_hit, sizeof(hit)) != cudaSuccess)
        return rc;
    if (!hit) return rc;
    const unsigned long long zero = 0;
    cudaMemcpyToSymbol(g_bounds_hit, &zero, sizeof(zero));
    const int site = (int)(hit >> 48) - 1;
    const long idx = (long)(hit & 0xFFFFFFFFFFFFull);
    return fail(c, DASHA_E_CUDA, std::string("bounds check: ") + (site >= 0 && site < BS_COUNT ? names[site] : "?") +
                                     " at node index " + std::to_string(idx));
}
#else
static int bounds_status(dasha_ctx*, int rc) { return rc; }
#endif
#ifndef DASHA_NO_TMA
// a bounded mbarrier wait of a TMA ring that ran out (the kernel returned early)
static int wait_status(dasha_ctx* c, int rc) {
    if (!c || !c->st) return rc;
    unsigned int hit = 0;
    if (cudaStreamSynchronize(c->st) != cudaSuccess || cudaMemcpyFromSymbol(&hit, g_wait_timeout, sizeof(hit)) != cudaSuccess)
        return rc;
    if (!hit) return rc;
    const unsigned int zero = 0;
    cudaMemcpyToSymbol(g_wait_timeout, &zero, sizeof(zero));
    return fail(c, DASHA_E_CUDA, "a TMA ring wait ran out (k_zpv_tma / k_zhydro_tma)");
}
#else
static int wait_status(dasha_ctx*, int rc) { return rc; }
#endif

template <class F>
static int host_call(dasha_ctx* c, F body) {
    try {
        return wait_status(c, bounds_status(c, body()));
    } catch (const std::bad_alloc&) {
        return fail(c, DASHA_E_NOMEM, "host allocation failed");
    } catch (const std::exception& e) {
        return fail(c, DASHA_E_INVALID, std::string("host error: ") + e.what());
    } catch (...) {
        return fail(c, DASHA_E_INVALID, "host error");
    }
}
template <class F>
static int engine_call(dasha_ctx* c, F call) {
    return host_call(c, [&] { return from_status(c, call()); });
}

extern "C" {

static int create_ctx(const dasha_grid_c* grid, const dasha_params_c* params, int nslabs, int slab, dasha_ctx** out);

int dasha_create(const dasha_grid_c* grid, const dasha_params_c* params, dasha_ctx** out) {
    return create_ctx(grid, params, 1, 0, out);
}

int dasha_slab_partition(int mz, int nslabs, int slab, int* first, int* count) {
    SlabPart sp;
    if (!first || !count || !slab_partition(mz, nslabs, slab, sp)) return DASHA_E_INVALID;
    *first = sp.first;
    *count = sp.count;
    return DASHA_OK;
}

int dasha_slab_halo_plan(int mz, int nslabs, int slab, long plane, int* peer, long* send_off, long* recv_off,
                         long* count) {
    SlabPart sp;
    if (!peer || !send_off || !recv_off || !count || plane < 1 || !slab_partition(mz, nslabs, slab, sp))
        return DASHA_E_INVALID;
    SlabGeom g;   // offsets in values: one byte per value
    g.n = nslabs; g.s = slab; g.mzl = sp.count + 4; g.sz = plane; g.elem = 1;
    peer[0] = g.lower() ? slab - 1 : -1;
    peer[1] = g.upper() ? slab + 1 : -1;
    send_off[0] = (long)g.send_lo(); recv_off[0] = (long)g.recv_lo();
    send_off[1] = (long)g.send_hi(); recv_off[1] = (long)g.recv_hi();
    *count = (long)g.span();
    return DASHA_OK;
}

int dasha_create_slab(const dasha_grid_c* grid, const dasha_params_c* params, int nslabs, int slab, dasha_ctx** out) {
    if (!out) return DASHA_E_INVALID;
    *out = nullptr;
    if (!grid || !params) return DASHA_E_INVALID;
    if (grid->periodic[0] == 0 && grid->periodic[1] == 0 && grid->periodic[2] == 0)
        return DASHA_E_UNSUPPORTED;   // the bounded configuration runs on one context
    SlabPart sp;
    if (!slab_partition(grid->mz, nslabs, slab, sp)) return DASHA_E_INVALID;
    return create_ctx(grid, params, nslabs, slab, out);
}

static int create_ctx(const dasha_grid_c* grid, const dasha_params_c* params, int nslabs, int slab, dasha_ctx** out) {
    if (!out) return DASHA_E_INVALID;
    *out = nullptr;
    if (!grid || !params || !grid->x || !grid->y || !grid->z) return DASHA_E_INVALID;
    if (grid->mx < 5 || grid->my < 5 || grid->mz < 7) return DASHA_E_INVALID;
    const bool bounded = grid->periodic[0] == 0 && grid->periodic[1] == 0 && grid->periodic[2] == 0;
    // rows move as 16-byte copies (4 FP32 or 2 FP64 values, row starts 16-byte aligned) and FP32
    // float pairs; the z-marching kernels take a narrower last x tile, except the viscous /
    // diffusive right-hand side (k_zst2), whose launch covers whole 32-node tiles
    if (!bounded && grid->mx % 4 != 0) return DASHA_E_UNSUPPORTED;
    const bool viscous = (params->viscos && params->mu != 0.0) || (params->diffu && (params->drho != 0.0 || params->dp != 0.0));
    if (!bounded && viscous && grid->mx % 32 != 0) return DASHA_E_UNSUPPORTED;
    if (!bounded && !(grid->periodic[0] == 1 && grid->periodic[1] == 1 && grid->periodic[2] == 0)) return DASHA_E_UNSUPPORTED;
    const dasha_params_c& p = *params;
    if (p.precision != 0 && p.precision != 1) return DASHA_E_INVALID;
    if (p.total_e != 1 || (!bounded && p.rcr > 0.0)) return DASHA_E_UNSUPPORTED;
    if (bounded && p.precision != 0) return DASHA_E_UNSUPPORTED;     // the bounded configuration is FP64
    if (p.uyzlimiter != 0 && p.uyzlimiter != 1) return DASHA_E_INVALID;
    if (!bounded && p.uyzlimiter) return DASHA_E_UNSUPPORTED;         // the limiter is a bounded-context option
    if (p.j0_mode != 0 && p.j0_mode != 1) return DASHA_E_INVALID;
    if (!(p.gamma > 1.0) || !(p.cfl > 0.0) || p.filter_every < 0) return DASHA_E_INVALID;
    dasha_ctx* c = new (std::nothrow) dasha_ctx();
    if (!c) return DASHA_E_NOMEM;
    try {
        c->mx = grid->mx; c->my = grid->my; c->mz = grid->mz;
        c->bounded = bounded;
        c->N = (long)c->mx * c->my * c->mz;
        c->P = p;
        c->ax.n = c->mx; c->ax.periodic = !bounded; c->ax.c.assign(grid->x, grid->x + c->mx);
        c->ay.n = c->my; c->ay.periodic = !bounded; c->ay.c.assign(grid->y, grid->y + c->my);
        c->az.n = c->mz; c->az.periodic = false; c->az.c.assign(grid->z, grid->z + c->mz);
        // a periodic axis continues with its first spacing across the wrap (t3dsdsc.f:278-283)
        c->ax.L = c->ax.c[c->mx - 1] - c->ax.c[0] + (c->ax.c[1] - c->ax.c[0]);
        c->ay.L = c->ay.c[c->my - 1] - c->ay.c[0] + (c->ay.c[1] - c->ay.c[0]);
        for (const Axis* a : {&c->ax, &c->ay, &c->az})
            for (int i = 0; i + 1 < a->n; ++i)
                if (!(a->c[i + 1] > a->c[i])) { delete c; return DASHA_E_INVALID; }
        if (cudaGetDevice(&c->device) != cudaSuccess) { delete c; return DASHA_E_CUDA; }
        if (cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) != cudaSuccess) { delete c; return DASHA_E_CUDA; }

        // host coefficient tables (FP64)
        HostTables H;
        H.mx = c->mx; H.my = c->my; H.mz = c->mz;
        const Axis* axes[3] = {&c->ax, &c->ay, &c->az};
        for (int d = 0; d < 3; ++d) {
            const Axis& a = *axes[d];
            int n = a.n;
            for (int q = 0; q < 8; ++q) H.coef[d][q].assign(n, 0.0);
            H.wp[d].assign(n, 0.0); H.wm[d].assign(n, 0.0);
            H.spacing[d].assign(n, 0.0); H.weight[d].assign(n, 0.0);
            for (int i = 0; i < n; ++i) {
                bool interior = a.periodic || (i >= 2 && i <= n - 3);
                if (interior) {
                    double x0 = a.at(i);
                    double hp1 = a.at(i + 1) - x0, hm1 = x0 - a.at(i - 1);
                    double hp2 = a.at(i + 2) - x0, hm2 = x0 - a.at(i - 2);
                    double w1[4], w2[4];
                    if (!stencil_weights(hp1, hm1, hp2, hm2, 1, w1) || !stencil_weights(hp1, hm1, hp2, hm2, 2, w2)) {
                        cudaStreamDestroy(c->st); delete c; return DASHA_E_INVALID;
                    }
                    for (int q = 0; q < 4; ++q) { H.coef[d][q][i] = w1[q]; H.coef[d][4 + q][i] = w2[q]; }
                }
                bool inner1 = a.periodic || (i >= 1 && i <= n - 2);
                if (inner1) {
                    double xm = a.at(i - 1), x0 = a.at(i), xp = a.at(i + 1);
                    H.wp[d][i] = 2.0 * (xp - x0) / (xp - xm);
                    H.wm[d][i] = 2.0 * (x0 - xm) / (xp - xm);
                }
                // forward spacing of node i (dxt of gridpntnew2), used by setdt
                H.spacing[d][i] = (a.periodic || i + 1 < n) ? a.at(i + 1) - a.at(i) : a.c[n - 1] - a.c[n - 2];
                // trapezoid volume weight
                if (a.periodic) H.weight[d][i] = 0.5 * (a.at(i + 1) - a.at(i - 1));
                else H.weight[d][i] = 0.5 * (a.c[std::min(i + 1, n - 1)] - a.c[std::max(i - 1, 0)]);
            }
            H.coord[d] = a.c;
        }
        H.cbx.assign(c->mx, 0.0);
        for (int i = 0; i < c->mx; ++i) H.cbx[i] = (1.0 / 32.0) * (1.0 - std::tanh((c->ax.c[i] + 3.0) / 8.0));

        if (nslabs > 1) {   // a z-slab: the local planes of every z table, the global grid's values
            SlabPart sp;
            slab_partition(c->mz, nslabs, slab, sp);
            const int z0 = sp.first - 2, mzl = sp.count + 4;
            auto cut = [&](std::vector<double>& v) { v = std::vector<double>(v.begin() + z0, v.begin() + z0 + mzl); };
            for (int q = 0; q < 8; ++q) cut(H.coef[2][q]);
            cut(H.wp[2]); cut(H.wm[2]); cut(H.spacing[2]); cut(H.weight[2]); cut(H.coord[2]);
            cut(c->az.c);
            c->nslabs = nslabs; c->slab = slab; c->zfirst = sp.first; c->mzg = c->mz;
            c->mz = mzl; c->az.n = mzl; H.mz = mzl;
            c->N = (long)c->mx * c->my * c->mz;
        } else {
            c->mzg = c->mz;
        }
        Status s;
        if (bounded) c->eng = make_engine_walls(c->mx, c->my, c->mz, p, c->st, grid->x, grid->y, grid->z, s);
        else if (p.precision == 0) c->eng = make_engine_f64(c->mx, c->my, c->mz, p, c->st, H, s);
        else c->eng = make_engine_f32(c->mx, c->my, c->mz, p, c->st, H, s);
        if (s.code != DASHA_OK) {
            int code = s.code;
            delete c->eng; c->eng = nullptr;
            cudaStreamDestroy(c->st);
            delete c;
            return code;
        }
    } catch (...) {
        if (c->eng) delete c->eng;
        if (c->st) cudaStreamDestroy(c->st);
        delete c;
        return DASHA_E_NOMEM;
    }
    if (c->slab > 0) c->eng->set_cfl_k0(2);   // planes 0 and 1 are the slab below's
    *out = c;
    return DASHA_OK;
}

void dasha_destroy(dasha_ctx* c) {
    if (!c) return;
    if (c->group) c->group->members[c->slab] = nullptr;
    if (c->eng) { cudaStreamSynchronize(c->st); delete c->eng; }
    c->halo.reset();
    if (c->st) cudaStreamDestroy(c->st);
    delete c;
}

const char* dasha_last_error(dasha_ctx* c) { return c ? c->err.c_str() : "null context"; }

// a z-slab takes the global grid's profiles (nprof arrays of mzg values, one after another)
// and keeps its own planes
static std::vector<double> slab_profiles(const dasha_ctx* c, const double* f, int nprof) {
    std::vector<double> v((size_t)nprof * c->mz);
    for (int m = 0; m < nprof; ++m)
        for (int k = 0; k < c->mz; ++k) v[(size_t)m * c->mz + k] = f[(size_t)m * c->mzg + (c->zfirst - 2) + k];
    return v;
}

// the profiles of the context's own planes
static int set_equilibrium_local(dasha_ctx* c, const double* rho0, const double* b0, const double* p0) {
    for (int k = 0; k < c->mz; ++k)
        if (!(rho0[k] > 0.0)) return fail(c, DASHA_E_INVALID, "rho0 must be positive");
    try {
        int rc = from_status(c, c->eng->set_equilibrium(rho0, b0, p0, nullptr));
        if (rc == DASHA_OK) c->eq_set = true;
        if (rc == DASHA_OK && c->bounded) c->state_set = true;    // the state initia leaves
        return rc;
    } catch (...) { return fail(c, DASHA_E_NOMEM, "host allocation failed"); }
}

int dasha_set_equilibrium(dasha_ctx* c, const double* rho0, const double* b0, const double* p0) {
    CAPI_GUARD(c);
    if (!rho0 || !b0 || !p0) return fail(c, DASHA_E_INVALID, "null equilibrium profile");
    if (!c->is_slab()) return set_equilibrium_local(c, rho0, b0, p0);
    return host_call(c, [&] {
        const std::vector<double> r = slab_profiles(c, rho0, 1), b = slab_profiles(c, b0, 3), q = slab_profiles(c, p0, 1);
        return set_equilibrium_local(c, r.data(), b.data(), q.data());
    });
}

int dasha_set_equilibrium_3d(dasha_ctx* c, const double* eq_f, long ld1, long ld2) {
    CAPI_GUARD(c);
    SLAB_UNSUPPORTED(c, "dasha_set_equilibrium_3d");
    if (!eq_f || ld1 < c->mx + 4 || ld2 < c->my) return fail(c, DASHA_E_INVALID, "bad equilibrium arguments");
    const int rc = engine_call(c, [&] { return c->eng->set_equilibrium_3d(eq_f, ld1, ld2); });
    if (rc == DASHA_OK) c->eq_set = true;
    if (rc == DASHA_OK && c->bounded) c->state_set = true;        // the state initia leaves
    return rc;
}

int dasha_set_equilibrium_current(dasha_ctx* c, const double* j0) {
    CAPI_GUARD(c);
    if (!j0) return fail(c, DASHA_E_INVALID, "null j0");
    if (!c->eq_set) return fail(c, DASHA_E_STATE, "set the equilibrium first");
    if (c->is_slab()) {
        return host_call(c, [&] {
            const std::vector<double> v = slab_profiles(c, j0, 3);
            return from_status(c, c->eng->set_j0(v.data()));
        });
    }
    return engine_call(c, [&] { return c->eng->set_j0(j0); });
}

static int check_ld(dasha_ctx* c, const void* p, long ld1, long ld2) {
    if (!p) return fail(c, DASHA_E_INVALID, "null host array");
    if (ld1 < c->mx + 4 || ld2 < c->my) return fail(c, DASHA_E_INVALID, "leading dimensions too small");
    return DASHA_OK;
}

int dasha_set_state(dasha_ctx* c, const double* x_f, long ld1, long ld2) {
    CAPI_GUARD(c);
    if (int rc = check_ld(c, x_f, ld1, ld2)) return rc;
    if (!c->eq_set) return fail(c, DASHA_E_STATE, "set the equilibrium before the state");
    int rc = engine_call(c, [&] { return c->eng->set_state(x_f, ld1, ld2); });
    if (rc == DASHA_OK) c->state_set = true;
    return rc;
}

int dasha_get_state(dasha_ctx* c, double* x_f, long ld1, long ld2) {
    CAPI_GUARD(c);
    if (int rc = check_ld(c, x_f, ld1, ld2)) return rc;
    if (!c->state_set) return fail(c, DASHA_E_STATE, "no state set");
    return engine_call(c, [&] { return c->eng->get_state(x_f, ld1, ld2); });
}

// Restart file of recrd / readin (t3dsdsc.f:4814-4861) streamed to or from the device state in
// z-plane chunks: record 2 is x(mx+4, my, mz+4, 8) in the reference's order, so each field is
// 2 planes of zero z halo, the mz planes of the chunks (each row with the periodic x halo
// copies that message4 leaves at a 1x1 process grid) and 2 more zero planes.
// The exact-resume record beside a restart file, <path>.state: the device state as stored, so
// that a run restored from it continues bit for bit (the reference's file holds FP64 totals,
// from which neither the FP64 perturbation split nor the FP32 pair (x, Kahan compensation) can
// be recovered exactly).  48-byte header: "DASHAST1", int32 precision, mx, my, mz, nfields,
// ncase, nstep, nst, double time; then nfields x mx*my*mz values of the context's type, node
// (i, j, k) at i + mx (j + my k), the 8 perturbation fields (rho - rho0, rho v, B - B0, p - p0)
// and in FP32 their 8 compensations.
static std::string state_record_path(const char* path) { return std::string(path) + ".state"; }
static void pack_state_header(unsigned char* h, const dasha_ctx* c, int nf, int ncase, int nstep, int nst, double time) {
    const int32_t v[8] = {c->P.precision, c->mx, c->my, c->mz, nf, ncase, nstep, nst};
    std::memcpy(h, "DASHAST1", 8);
    std::memcpy(h + 8, v, sizeof(v));
    std::memcpy(h + 40, &time, sizeof(double));
}

int dasha_checkpoint(dasha_ctx* c, const char* path, int ncase, int nstep, double time, int nst,
                     long max_subrecord) {
    CAPI_GUARD(c);
    SLAB_UNSUPPORTED(c, "dasha_checkpoint");
    if (!path || max_subrecord < 0) return fail(c, DASHA_E_INVALID, "bad checkpoint arguments");
    if (!c->state_set) return fail(c, DASHA_E_STATE, "no state set");
    return host_call(c, [&]() -> int {
        const long maxsub = max_subrecord == 0 ? kMaxSubrecord : std::min(max_subrecord, kMaxSubrecord);
        File f(path, "wb");
        if (!f.f) return fail(c, DASHA_E_INVALID, std::string("cannot open ") + path);
        const int mx = c->mx, my = c->my, mz = c->mz;
        const long row = mx + 4;
        unsigned char hdr[20];
        pack_restart_header(hdr, ncase, nstep, time, nst);
        RecWriter w1(f.f, 20, maxsub);
        w1.put(hdr, 20);
        if (!w1.finish()) return fail(c, DASHA_E_INVALID, std::string("writing ") + path + " failed");
        RecWriter w(f.f, (long)sizeof(double) * row * my * (mz + 4) * 8, maxsub);
        std::vector<double> rb(row), zero(row, 0.0);
        auto zplanes = [&]() { for (long r = 0; r < 2L * my && w.ok; ++r) w.put(zero.data(), (long)sizeof(double) * row); };
        const int rc = from_status(c, c->eng->state_out([&](int, int k0, int k1, const double* rows) {
            if (k0 == 0) zplanes();
            for (long r = 0; r < (long)(k1 - k0) * my && w.ok; ++r) {
                const double* v = rows + r * mx;
                rb[0] = v[mx - 2]; rb[1] = v[mx - 1];
                std::memcpy(rb.data() + 2, v, sizeof(double) * mx);
                rb[mx + 2] = v[0]; rb[mx + 3] = v[1];
                w.put(rb.data(), (long)sizeof(double) * row);
            }
            if (k1 == mz) zplanes();
            return w.ok;
        }));
        if (rc != DASHA_OK) return rc;
        const bool ok = w.finish();
        if (!f.close() || !ok) return fail(c, DASHA_E_INVALID, std::string("writing ") + path + " failed");
        // the exact-resume record
        const std::string sp = state_record_path(path);
        File g(sp.c_str(), "wb");
        if (!g.f) return fail(c, DASHA_E_INVALID, "cannot open " + sp);
        unsigned char h[48];
        pack_state_header(h, c, c->eng->raw_fields(), ncase, nstep, nst, time);
        bool gok = std::fwrite(h, 1, 48, g.f) == 48;
        const int rc3 = from_status(c, c->eng->raw_out([&](const void* p, size_t n) {
            gok = gok && std::fwrite(p, 1, n, g.f) == n;
            return gok;
        }));
        if (rc3 != DASHA_OK) return rc3;
        if (!g.close() || !gok) return fail(c, DASHA_E_INVALID, "writing " + sp + " failed");
        return DASHA_OK;
    });
}

int dasha_restore(dasha_ctx* c, const char* path, int* ncase, int* nstep, double* time, int* nst) {
    CAPI_GUARD(c);
    SLAB_UNSUPPORTED(c, "dasha_restore");
    if (!path || !ncase || !nstep || !time || !nst) return fail(c, DASHA_E_INVALID, "bad restore arguments");
    if (!c->eq_set) return fail(c, DASHA_E_STATE, "set the equilibrium before the state");
    bool touched = false;   // set once the device state starts to change
    const int rc = host_call(c, [&]() -> int {
        File f(path, "rb");
        if (!f.f) return fail(c, DASHA_E_INVALID, std::string("cannot open ") + path);
        const int mx = c->mx, my = c->my, mz = c->mz;
        const long row = mx + 4, total = (long)sizeof(double) * row * my * (mz + 4) * 8;
        unsigned char hdr[20];
        RecReader r1(f.f, 20);
        r1.get(hdr, 20);
        // the markers of record 2 are checked before the device state is touched
        if (!r1.finish() || !scan_record(f.f, total))
            return fail(c, DASHA_E_INVALID, std::string(path) + " is not a restart file of this grid");
        // an exact-resume record beside the file must belong to it: checked before the state
        // is touched
        int h_ncase, h_nstep, h_nst;
        double h_time;
        unpack_restart_header(hdr, &h_ncase, &h_nstep, &h_time, &h_nst);
        const std::string sp = state_record_path(path);
        File g(sp.c_str(), "rb");
        const size_t raw_bytes = c->eng->raw_elem() * (size_t)c->eng->raw_fields() * (size_t)mx * my * mz;
        if (g.f) {
            unsigned char h[48], want[48];
            pack_state_header(want, c, c->eng->raw_fields(), h_ncase, h_nstep, h_nst, h_time);
            std::fseek(g.f, 0, SEEK_END);
            const long len = std::ftell(g.f);
            std::fseek(g.f, 0, SEEK_SET);
            if (std::fread(h, 1, 48, g.f) != 48 || std::memcmp(h, want, 48) != 0 || len != (long)(48 + raw_bytes))
                return fail(c, DASHA_E_INVALID, sp + " does not belong to " + path + " and this context");
        }
        RecReader r(f.f, total);
        std::vector<double> rb(row), skip(row);
        auto zplanes = [&]() { for (long q = 0; q < 2L * my && r.ok; ++q) r.get(skip.data(), (long)sizeof(double) * row); };
        touched = true;
        const int rc2 = from_status(c, c->eng->state_in([&](int, int k0, int k1, double* rows) {
            if (k0 == 0) zplanes();
            for (long q = 0; q < (long)(k1 - k0) * my && r.ok; ++q) {
                r.get(rb.data(), (long)sizeof(double) * row);
                std::memcpy(rows + q * mx, rb.data() + 2, sizeof(double) * mx);
            }
            if (k1 == mz) zplanes();
            return r.ok;
        }));
        if (rc2 != DASHA_OK) return rc2;
        if (!r.finish()) return fail(c, DASHA_E_INVALID, std::string("reading ") + path + " failed");
        if (g.f) {   // the state exactly as it was stored
            bool gok = true;
            const int rc3 = from_status(c, c->eng->raw_in([&](void* p, size_t n) {
                gok = gok && std::fread(p, 1, n, g.f) == n;
                return gok;
            }));
            if (rc3 != DASHA_OK) return rc3;
        }
        unpack_restart_header(hdr, ncase, nstep, time, nst);
        return DASHA_OK;
    });
    if (rc == DASHA_OK) c->state_set = true;
    else if (touched) c->state_set = false;   // part of the state may have been replaced
    return rc;
}

int dasha_stream_out(dasha_ctx* c, int what, dasha_chunk_fn fn, void* user) {
    CAPI_GUARD(c);
    SLAB_UNSUPPORTED(c, "dasha_stream_out");
    if (!fn || (what != 0 && what != 1)) return fail(c, DASHA_E_INVALID, "bad stream arguments");
    if (!c->state_set) return fail(c, DASHA_E_STATE, "no state set");
    return engine_call(c, [&] {
        const ChunkOut take = [&](int m, int k0, int k1, const double* rows) { return fn(user, m, k0, k1, rows) == 0; };
        return what == 0 ? c->eng->state_out(take) : c->eng->current_out(take);
    });
}

// m3d of recrd3 (t3dsdsc.f:5365-5402) from the context: the state's fields stream in order
// (rho kept on the host for v = (rho v)/rho), then the current's, each list formatted while the
// next chunk's transfer runs; the text equals dasha_m3d_write of the get_state / current arrays.
int dasha_m3d_write_ctx(dasha_ctx* c, const char* path, double time) {
    CAPI_GUARD(c);
    SLAB_UNSUPPORTED(c, "dasha_m3d_write_ctx");
    if (!path) return fail(c, DASHA_E_INVALID, "null path");
    if (!c->state_set) return fail(c, DASHA_E_STATE, "no state set");
    return host_call(c, [&]() -> int {
        File f(path, "w");
        if (!f.f) return fail(c, DASHA_E_INVALID, std::string("cannot open ") + path);
        const int mx = c->mx, my = c->my, mz = c->mz;
        const int hdr[4] = {3, mx, my, mz};
        ld_ints(f.f, hdr, 4);
        ld_real(f.f, time);
        bool ok = write_list(f.f, (long)mx + my + mz, 11, 10, 4, 0, [&](long n) {
            return n < mx ? c->ax.c[n] : (n < (long)mx + my ? c->ay.c[n - mx] : c->az.c[n - mx - my]);
        });
        if (!ok) return fail(c, DASHA_E_INVALID, std::string("writing ") + path + " failed");
        std::vector<double> rho((size_t)c->N);
        ListWriter lw(f.f, 11, 10, 4, 0);
        int open_q = -1;
        auto list = [&](int q, int k0, int k1, const double* rows) {
            if (q != open_q) {               // a new field: close the last list, number the next
                if (open_q >= 0) lw.end();
                const int iq = q + 1;
                ld_ints(f.f, &iq, 1);
                open_q = q;
            }
            const long cnt = (long)(k1 - k0) * mx * my;
            const size_t off = (size_t)k0 * mx * my;
            if (q == 0) std::memcpy(rho.data() + off, rows, sizeof(double) * cnt);
            if (q >= 1 && q <= 3) lw.put(cnt, [&](long n) { return rows[n] / rho[off + n]; });
            else lw.put(cnt, [&](long n) { return rows[n]; });
            return lw.ok;
        };
        int rc = from_status(c, c->eng->state_out([&](int m, int k0, int k1, const double* rows) {
            return list(m, k0, k1, rows);
        }));
        if (rc == DASHA_OK)
            rc = from_status(c, c->eng->current_out([&](int m, int k0, int k1, const double* rows) {
                return list(8 + m, k0, k1, rows);
            }));
        if (rc != DASHA_OK) return rc;
        ok = lw.end();
        if (!f.close() || !ok) return fail(c, DASHA_E_INVALID, std::string("writing ") + path + " failed");
        return DASHA_OK;
    });
}

// the reference's two stop conditions of the step loop on a new dt (t3dsdsc.f:142-154, 1232)
static int setdt_guards(dasha_ctx* c, double dt, int blowup) {
    if (blowup) return fail(c, DASHA_E_BLOWUP, "max Jy on the mid-y plane reached 1e7 (or is not finite)");
    if (!(dt > 0.0) || !std::isfinite(dt)) return fail(c, DASHA_E_DT_COLLAPSE, "dt is not a positive finite number");
    if (!c->have_dt0) { c->dt0 = dt; c->have_dt0 = true; }
    else if (dt < 0.1 * c->dt0) return fail(c, DASHA_E_DT_COLLAPSE, "dt fell below 0.1*dt0");
    return DASHA_OK;
}

int dasha_setdt(dasha_ctx* c, double time, double* dt_out) {
    CAPI_GUARD(c);
    if (int rc = slab_single_call(c)) return rc;
    (void)time;
    if (!dt_out) return fail(c, DASHA_E_INVALID, "null dt_out");
    if (!c->state_set) return fail(c, DASHA_E_STATE, "no state set");
    int blowup = 0;
    double dt = 0.;
    int rc = engine_call(c, [&] { return c->eng->setdt(&dt, &blowup); });
    if (rc) return rc;
    *dt_out = dt;
    return setdt_guards(c, dt, blowup);
}

int dasha_stepon(dasha_ctx* c, double time, double dt, int nstep) {
    CAPI_GUARD(c);
    if (int rc = slab_single_call(c)) return rc;
    if (!c->state_set) return fail(c, DASHA_E_STATE, "no state set");
    if (!(dt > 0.0) || !std::isfinite(dt)) return fail(c, DASHA_E_INVALID, "dt must be positive and finite");
    return engine_call(c, [&] { return c->eng->stepon(time, dt, nstep); });
}

int dasha_current(dasha_ctx* c, double* cur_f, long ld1, long ld2) {
    CAPI_GUARD(c);
    if (int rc = slab_single_call(c)) return rc;
    if (int rc = check_ld(c, cur_f, ld1, ld2)) return rc;
    if (!c->state_set) return fail(c, DASHA_E_STATE, "no state set");
    return engine_call(c, [&] { return c->eng->current(cur_f, ld1, ld2); });
}

int dasha_midplane(dasha_ctx* c, double* plane) {
    CAPI_GUARD(c);
    SLAB_UNSUPPORTED(c, "dasha_midplane");
    if (!plane) return fail(c, DASHA_E_INVALID, "null plane");
    if (!c->state_set) return fail(c, DASHA_E_STATE, "no state set");
    return engine_call(c, [&] { return c->eng->midplane(plane); });
}

int dasha_rhs(dasha_ctx* c, double t, double* xdif_f, long ld1, long ld2) {
    CAPI_GUARD(c);
    SLAB_UNSUPPORTED(c, "dasha_rhs");
    if (int rc = check_ld(c, xdif_f, ld1, ld2)) return rc;
    if (!c->state_set) return fail(c, DASHA_E_STATE, "no state set");
    return engine_call(c, [&] { return c->eng->rhs(t, xdif_f, ld1, ld2); });
}

int dasha_diagnostics(dasha_ctx* c, double* out) {
    CAPI_GUARD(c);
    if (int rc = slab_single_call(c)) return rc;
    if (!out) return fail(c, DASHA_E_INVALID, "null out");
    if (!c->state_set) return fail(c, DASHA_E_STATE, "no state set");
    return engine_call(c, [&] { return c->eng->diagnostics(out); });
}

int dasha_adjoint_flux_grad(dasha_ctx* c, int nsteps, const double* dt_seq, int snaps, double* dPhi_deta,
                            double* dPhi_dpsi) {
    CAPI_GUARD(c);
    SLAB_UNSUPPORTED(c, "dasha_adjoint_flux_grad");
    if (nsteps < 0 || (nsteps > 0 && !dt_seq) || snaps < 0 || !dPhi_deta || !dPhi_dpsi)
        return fail(c, DASHA_E_INVALID, "bad adjoint arguments");
    if (!c->state_set) return fail(c, DASHA_E_STATE, "no state set");
    if (c->P.precision != 0) return fail(c, DASHA_E_UNSUPPORTED, "the adjoint runs on FP64 contexts only");
    return engine_call(c, [&] { return c->eng->adjoint_flux_grad(nsteps, dt_seq, snaps, dPhi_deta, dPhi_dpsi); });
}

int dasha_adjoint_rhs(dasha_ctx* c, const double* w_f, double* out_f, long ld1, long ld2) {
    CAPI_GUARD(c);
    SLAB_UNSUPPORTED(c, "dasha_adjoint_rhs");
    if (int rc = check_ld(c, w_f, ld1, ld2)) return rc;
    if (int rc = check_ld(c, out_f, ld1, ld2)) return rc;
    if (!c->state_set) return fail(c, DASHA_E_STATE, "no state set");
    return engine_call(c, [&] { return c->eng->adjoint_rhs(w_f, out_f, ld1, ld2); });
}

int dasha_timer(dasha_ctx* c, int op, double* ms) {
    CAPI_GUARD(c);
    EngineBase* e = c->eng;
    if (!e->t0) {
        if (cudaEventCreate(&e->t0) != cudaSuccess || cudaEventCreate(&e->t1) != cudaSuccess)
            return fail(c, DASHA_E_CUDA, "cudaEventCreate failed");
    }
    if (op == 0) {
        if (cudaEventRecord(e->t0, c->st) != cudaSuccess) return fail(c, DASHA_E_CUDA, "cudaEventRecord failed");
        return DASHA_OK;
    }
    if (op != 1 || !ms) return fail(c, DASHA_E_INVALID, "dasha_timer: op must be 0 or 1 (with ms)");
    if (cudaEventRecord(e->t1, c->st) != cudaSuccess || cudaEventSynchronize(e->t1) != cudaSuccess)
        return fail(c, DASHA_E_CUDA, "cudaEventSynchronize failed");
    float f = 0.f;
    if (cudaEventElapsedTime(&f, e->t0, e->t1) != cudaSuccess) return fail(c, DASHA_E_CUDA, "cudaEventElapsedTime failed");
    *ms = f;
    return DASHA_OK;
}

int dasha_profile(dasha_ctx* c, int enable) {
    CAPI_GUARD(c);
    c->eng->prof.on = enable != 0;
    return DASHA_OK;
}

int dasha_profile_read(dasha_ctx* c, int* n, char* names, double* ms, long* launches, double* bytes) {
    CAPI_GUARD(c);
    if (!n || *n < 0 || (*n > 0 && (!names || !ms || !launches || !bytes))) return fail(c, DASHA_E_INVALID, "bad arguments");
    Profiler& p = c->eng->prof;
    if (cudaStreamSynchronize(c->st) != cudaSuccess) return fail(c, DASHA_E_CUDA, "stream synchronize failed");
    size_t nt = p.names.size();
    std::vector<double> tot(nt, 0.0);
    std::vector<long> cnt(nt, 0);
    for (auto& r : p.recs) {
        float f = 0.f;
        cudaEventElapsedTime(&f, r.a, r.b);
        tot[r.tag] += f;
        cnt[r.tag] += 1;
    }
    int rows = (int)std::min<size_t>(nt, (size_t)*n);
    for (int q = 0; q < rows; ++q) {
        std::memset(names + 32 * q, 0, 32);
        std::strncpy(names + 32 * q, p.names[q].c_str(), 31);
        ms[q] = tot[q]; launches[q] = cnt[q]; bytes[q] = p.bytes[q];
    }
    *n = (int)nt;
    p.recs.clear();
    p.used = 0;
    return DASHA_OK;
}

// ---- z-slab groups (halo.h) ----

int dasha_slab_rows(dasha_ctx* c, int* first, int* count, int* mz_local) {
    CAPI_GUARD(c);
    if (!first || !count || !mz_local) return fail(c, DASHA_E_INVALID, "null argument");
    *first = c->zfirst;
    *count = c->mz - 4;
    *mz_local = c->mz;
    return DASHA_OK;
}

}  // extern "C"

// the slab s of every context is ctxs[s]: one grid, parameters and precision
static int check_group(dasha_ctx* const* cs, int n) {
    if (!cs || n < 2) return DASHA_E_INVALID;
    for (int s = 0; s < n; ++s) {
        const dasha_ctx* c = cs[s];
        if (!c || c->nslabs != n || c->slab != s || c->mx != cs[0]->mx || c->my != cs[0]->my ||
            c->mzg != cs[0]->mzg || c->P.precision != cs[0]->P.precision)
            return DASHA_E_INVALID;
        if (c->sticky) return c->sticky;
    }
    return DASHA_OK;
}

// runs body(ctx, s) for every slab of a linked group, one host thread per slab with its device
// current; a slab that fails releases the others from the group's barriers
template <class F>
static int group_run(dasha_ctx* const* cs, int n, F body);

extern "C" {

int dasha_slab_link(dasha_ctx* const* cs, int n) {
    if (int rc = check_group(cs, n)) return rc;
    for (int s = 0; s < n; ++s)
        if (cs[s]->halo) return fail(cs[s], DASHA_E_STATE, "slab already joined to a group");
    try {
        auto grp = std::make_shared<LocalGroup>(n);
        std::vector<std::unique_ptr<Halo>> hs;
        for (int s = 0; s < n; ++s) {
            auto h = std::make_unique<HaloLocal>(grp);
            h->geo = cs[s]->eng->slab_geom();
            h->geo.n = n; h->geo.s = s; h->geo.device = cs[s]->device;
            h->geo.zfirst = cs[s]->zfirst; h->geo.mzg = cs[s]->mzg;
            hs.push_back(std::move(h));
        }
        // neighbours on different GPUs copy over NVLink: peer access both ways where the pair has it
        int cur = 0;
        cudaGetDevice(&cur);
        for (int s = 0; s + 1 < n; ++s) {
            const int a = cs[s]->device, b = cs[s + 1]->device;
            if (a == b) continue;
            int ab = 0, ba = 0;
            cudaDeviceCanAccessPeer(&ab, a, b);
            cudaDeviceCanAccessPeer(&ba, b, a);
            if (ab && cudaSetDevice(a) == cudaSuccess && cudaDeviceEnablePeerAccess(b, 0) != cudaSuccess) cudaGetLastError();
            if (ba && cudaSetDevice(b) == cudaSuccess && cudaDeviceEnablePeerAccess(a, 0) != cudaSuccess) cudaGetLastError();
        }
        cudaSetDevice(cur);
        for (int s = 0; s < n; ++s) {
            grp->members[s] = &hs[s]->geo;
            cs[s]->halo = std::move(hs[s]);
            cs[s]->eng->halo = cs[s]->halo.get();
            cs[s]->group = grp;
        }
    } catch (...) {
        return DASHA_E_NOMEM;
    }
    return DASHA_OK;
}

}  // extern "C"

template <class F>
static int group_run(dasha_ctx* const* cs, int n, F body) {
    if (int rc = check_group(cs, n)) return rc;
    std::shared_ptr<LocalGroup> grp = cs[0]->group;
    for (int s = 0; s < n; ++s)
        if (!cs[s]->group || cs[s]->group != grp) return fail(cs[s], DASHA_E_STATE, "slabs not linked as one group");
    grp->bar.reset();
    std::vector<int> rc(n, DASHA_OK);
    std::vector<std::thread> th;
    bool started = true;
    try {
        for (int s = 0; s < n; ++s)
            th.emplace_back([&, s] {
                if (cudaSetDevice(cs[s]->device) != cudaSuccess) rc[s] = fail(cs[s], DASHA_E_CUDA, "cudaSetDevice failed");
                else rc[s] = body(cs[s], s);
                if (rc[s]) grp->bar.fail();
            });
    } catch (...) {
        started = false;    // a thread could not start: the started ones leave the barriers
        grp->bar.fail();
    }
    for (auto& t : th) t.join();
    if (!started) return DASHA_E_NOMEM;
    for (int s = 0; s < n; ++s)   // the first slab's own failure, not the others' release
        if (rc[s] && cs[s]->halo && cs[s]->err.find("halo exchange") == std::string::npos) return rc[s];
    for (int s = 0; s < n; ++s)
        if (rc[s]) return rc[s];
    return DASHA_OK;
}

extern "C" {

int dasha_group_setdt(dasha_ctx* const* cs, int n, double time, double* dt_out) {
    (void)time;
    if (!dt_out) return DASHA_E_INVALID;
    if (int rc = check_group(cs, n)) return rc;
    for (int s = 0; s < n; ++s)
        if (!cs[s]->state_set) return fail(cs[s], DASHA_E_STATE, "no state set");
    std::vector<double> dt(n, 0.0);
    std::vector<int> bl(n, 0);
    int rc = group_run(cs, n, [&](dasha_ctx* c, int s) { return engine_call(c, [&] { return c->eng->setdt(&dt[s], &bl[s]); }); });
    if (rc) return rc;
    double d = dt[0];
    int b = bl[0];
    for (int s = 1; s < n; ++s) {   // the smallest dt (a NaN wins), any blow-up
        d = (d != d || dt[s] != dt[s]) ? (d != d ? d : dt[s]) : std::fmin(d, dt[s]);
        b |= bl[s];
    }
    *dt_out = d;
    for (int s = 1; s < n; ++s) { cs[s]->have_dt0 = cs[0]->have_dt0; cs[s]->dt0 = cs[0]->dt0; }
    rc = setdt_guards(cs[0], d, b);
    for (int s = 1; s < n; ++s) { cs[s]->have_dt0 = cs[0]->have_dt0; cs[s]->dt0 = cs[0]->dt0; }
    return rc;
}

int dasha_group_stepon(dasha_ctx* const* cs, int n, double time, double dt, int nstep) {
    if (int rc = check_group(cs, n)) return rc;
    if (!(dt > 0.0) || !std::isfinite(dt)) return DASHA_E_INVALID;
    for (int s = 0; s < n; ++s)
        if (!cs[s]->state_set) return fail(cs[s], DASHA_E_STATE, "no state set");
    return group_run(cs, n, [&](dasha_ctx* c, int) { return engine_call(c, [&] { return c->eng->stepon(time, dt, nstep); }); });
}

int dasha_group_current(dasha_ctx* const* cs, int n, double* const* cur_f, long ld1, long ld2) {
    if (int rc = check_group(cs, n)) return rc;
    if (!cur_f) return DASHA_E_INVALID;
    for (int s = 0; s < n; ++s) {
        if (int rc = check_ld(cs[s], cur_f[s], ld1, ld2)) return rc;
        if (!cs[s]->state_set) return fail(cs[s], DASHA_E_STATE, "no state set");
    }
    return group_run(cs, n, [&](dasha_ctx* c, int s) { return engine_call(c, [&] { return c->eng->current(cur_f[s], ld1, ld2); }); });
}

int dasha_group_diagnostics(dasha_ctx* const* cs, int n, double* out) {
    if (int rc = check_group(cs, n)) return rc;
    if (!out) return DASHA_E_INVALID;
    for (int s = 0; s < n; ++s)
        if (!cs[s]->state_set) return fail(cs[s], DASHA_E_STATE, "no state set");
    std::vector<double> part((size_t)n * DASHA_NDIAG, 0.0);
    int rc = group_run(cs, n, [&](dasha_ctx* c, int s) {
        return engine_call(c, [&] { return c->eng->diagnostics(part.data() + (size_t)s * DASHA_NDIAG); });
    });
    if (rc) return rc;
    for (int q = 0; q < DASHA_NDIAG; ++q) out[q] = part[q];
    for (int s = 1; s < n; ++s) {   // sums of mass, energy, flux; extrema of J
        const double* p = part.data() + (size_t)s * DASHA_NDIAG;
        for (int q = 0; q < 3; ++q) out[q] += p[q];
        for (int q = 3; q < 9; q += 2) { out[q] = std::fmax(out[q], p[q]); out[q + 1] = std::fmin(out[q + 1], p[q + 1]); }
    }
    return DASHA_OK;
}

int dasha_nccl_unique_id(void* id, int nbytes) {
    if (!id || nbytes < (int)sizeof(ncclUniqueId)) return DASHA_E_INVALID;
    const NcclApi& a = NcclApi::get();
    if (!a.ok()) return DASHA_E_UNSUPPORTED;
    ncclUniqueId u;
    if (a.get_unique_id(&u) != ncclSuccess) return DASHA_E_CUDA;
    std::memcpy(id, &u, sizeof(u));
    return DASHA_OK;
}

int dasha_slab_nccl(dasha_ctx* c, const void* id, int nbytes) {
    CAPI_GUARD(c);
    if (!id || nbytes < (int)sizeof(ncclUniqueId)) return fail(c, DASHA_E_INVALID, "the NCCL id is 128 bytes");
    if (c->halo) return fail(c, DASHA_E_STATE, "slab already joined");
    return host_call(c, [&] {
        auto h = std::make_unique<HaloNccl>();
        h->geo = c->eng->slab_geom();
        h->geo.n = c->nslabs; h->geo.s = c->slab; h->geo.device = c->device;
        h->geo.zfirst = c->zfirst; h->geo.mzg = c->mzg;
        ncclUniqueId u;
        std::memcpy(&u, id, sizeof(u));
        if (cudaSetDevice(c->device) != cudaSuccess) return fail(c, DASHA_E_CUDA, "cudaSetDevice failed");
        if (!h->init(u)) return fail(c, NcclApi::get().ok() ? DASHA_E_CUDA : DASHA_E_UNSUPPORTED, h->err);
        c->halo = std::move(h);
        c->eng->halo = c->halo.get();
        return (int)DASHA_OK;
    });
}

}  // extern "C"
