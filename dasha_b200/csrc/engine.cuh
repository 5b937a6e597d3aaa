// engine.cuh -- device buffers and the launch sequence of one RK4 step (stepon, right,
// current, setdt, diagn of t3dsdsc.f), templated on the storage type (double / float).
#pragma once
#include "dasha_capi.h"
#include "mhd_kernels.cuh"
#include "zm_kernels.cuh"
#include "zpv.cuh"
#include "zpv2.cuh"
#include "zcurl.cuh"
#include "zhydro.cuh"
#include "zeh.cuh"
#include "adjoint.cuh"
#include "checkpoint_schedule.h"
#include "halo.h"
#include "host_pool.h"
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <cstdlib>
#include <type_traits>
#include <string>
#include <vector>
#include <cmath>
#include <cstring>
#include <algorithm>
#include <thread>
#include <functional>

namespace dasha {

struct Status {
    int code = 0;
    std::string msg;
    static Status ok() { return Status(); }
    static Status err(int c, const std::string& m) { Status s; s.code = c; s.msg = m; return s; }
};

#define DASHA_CK(call)                                                                         \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            return Status::err(DASHA_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// FP64 host tables built by dasha_create: per axis d (0=x,1=y,2=z)
struct HostTables {
    int mx, my, mz;
    std::vector<double> coef[3][8];   // a1 b1 c1 d1 a2 b2 c2 d2
    std::vector<double> wp[3], wm[3]; // difc weights
    std::vector<double> spacing[3];   // forward spacing (setdt)
    std::vector<double> weight[3];    // trapezoid weights (diagnostics)
    std::vector<double> coord[3];
    std::vector<double> cbx;          // (1/32)(1 - tanh((x+3)/8))
};

// Optional per-launch CUDA-event profiler (dasha_profile).
struct Profiler {
    bool on = false;
    struct Rec { int tag; cudaEvent_t a, b; };
    std::vector<Rec> recs;
    std::vector<std::string> names;
    std::vector<double> bytes;
    std::vector<cudaEvent_t> pool;
    size_t used = 0;
    int tag_of(const char* name, double b) {
        for (size_t q = 0; q < names.size(); ++q) if (names[q] == name) return (int)q;
        names.push_back(name); bytes.push_back(b);
        return (int)names.size() - 1;
    }
    cudaEvent_t ev() {
        if (used == pool.size()) { cudaEvent_t e; cudaEventCreate(&e); pool.push_back(e); }
        return pool[used++];
    }
    ~Profiler() { for (auto e : pool) cudaEventDestroy(e); }
};

// Host work on one chunk of a state transfer: field m on z planes k0..k1-1 as (k1-k0)*my rows
// of mx FP64 values, x fastest; false stops the transfer.
using ChunkIn = std::function<bool(int m, int k0, int k1, double* rows)>;
using ChunkOut = std::function<bool(int m, int k0, int k1, const double* rows)>;

struct EngineBase {
    Profiler prof;
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    // z-slab contexts (halo.h): the ghost-plane exchange, owned by the context; null otherwise
    Halo* halo = nullptr;
    // the slab's pool layout for the exchange, and the first plane of its setdt region
    virtual SlabGeom slab_geom() const { return SlabGeom(); }
    virtual void set_cfl_k0(int) {}
    virtual ~EngineBase() {
        if (t0) cudaEventDestroy(t0);
        if (t1) cudaEventDestroy(t1);
    }
    virtual Status set_equilibrium(const double* rho0, const double* b0, const double* p0, const double* j0) = 0;
    virtual Status set_j0(const double* j0) = 0;
    // a 3-D equilibrium (rho0, B0, p0 as 5 fields in the state layout): bounded contexts only
    virtual Status set_equilibrium_3d(const double*, long, long) {
        return Status::err(DASHA_E_UNSUPPORTED, "a 3-D equilibrium needs a bounded (periodic 0,0,0) context");
    }
    virtual Status set_state(const double* x, long ld1, long ld2) = 0;
    virtual Status get_state(double* x, long ld1, long ld2) = 0;
    virtual Status state_in(const ChunkIn& fill) = 0;
    virtual Status state_out(const ChunkOut& take) = 0;
    virtual Status current_out(const ChunkOut& take) = 0;
    // The device state as stored (the perturbation fields, and in FP32 their Kahan
    // compensations after them), raw bytes in node order, in pieces of at most 64 MB: out hands
    // each piece to `take`, in fills each piece from `give` and replaces the state only whole
    // (the fields arrive in a spare buffer first).
    virtual int raw_fields() const = 0;
    virtual size_t raw_elem() const = 0;
    virtual Status raw_out(const std::function<bool(const void*, size_t)>& take) = 0;
    virtual Status raw_in(const std::function<bool(void*, size_t)>& give) = 0;
    virtual Status setdt(double* dt, int* blowup) = 0;
    virtual Status stepon(double time, double dt, int nstep) = 0;
    virtual Status current(double* cur, long ld1, long ld2) = 0;
    virtual Status midplane(double* out) = 0;
    virtual Status rhs(double t, double* xdif, long ld1, long ld2) = 0;
    virtual Status diagnostics(double* out) = 0;
    virtual Status adjoint_flux_grad(int nsteps, const double* dt_seq, int snaps, double* deta, double* dpsi) = 0;
    virtual Status adjoint_rhs(const double* w, double* out, long ld1, long ld2) = 0;
};

EngineBase* make_engine_f64(int mx, int my, int mz, const dasha_params_c& p, cudaStream_t st, const HostTables& H,
                            Status& s);
EngineBase* make_engine_f32(int mx, int my, int mz, const dasha_params_c& p, cudaStream_t st, const HostTables& H,
                            Status& s);
// the reference's bounded configuration (walls.cu): periodic = {0, 0, 0}, FP64
EngineBase* make_engine_walls(int mx, int my, int mz, const dasha_params_c& p, cudaStream_t st, const double* x,
                              const double* y, const double* z, Status& s);

// Launch with optional event bracketing; bytes = algorithmic bytes of the launch.
// Every launch is also an NVTX range named by its tag (a no-op unless a tool such as nsys or
// ncu --nvtx is attached), so a timeline or a capture filter sees the step's structure.
#define DASHA_LAUNCH(tag, bytes, ...)                                                          \
    do {                                                                                       \
        int tg_ = -1;                                                                          \
        cudaEvent_t a_ = nullptr;                                                              \
        nvtxRangePushA(tag);                                                                   \
        if (prof.on) { tg_ = prof.tag_of(tag, (double)(bytes)); a_ = prof.ev(); cudaEventRecord(a_, st); } \
        __VA_ARGS__;                                                                           \
        if (prof.on) { cudaEvent_t b_ = prof.ev(); cudaEventRecord(b_, st); prof.recs.push_back({tg_, a_, b_}); } \
        nvtxRangePop();                                                                        \
    } while (0)

#ifndef DASHA_NO_TMA
// cuTensorMapEncodeTiled through the runtime's driver entry point (no link against libcuda)
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
inline EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return (EncodeTiledFn) nullptr;
        return reinterpret_cast<EncodeTiledFn>(f);
    }();
    return fn;
}
#endif

// an NVTX range over a scope: the reference routine a group of launches stands for
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

// host transfer chunks and equilibrium profile lookup (defined after Engine)
template <class T>
__global__ void k_import_chunk(int mx, int my, int k0, const double* src, const double* eqprof, T* dst);
template <class T>
__global__ void k_export_chunk(int mx, int my, int k0, const T* src, const T* comp, const double* eqprof, double* dst);
template <class T>
__global__ void k_midplane(Geo<T> g, int j, F8<T> x, F8<T> comp, F3<T> cur, double* out);
template <class T>
inline const double* eq_profile(const Geo<T>& g, int m);

template <class T>
class Engine : public EngineBase {
public:
    static constexpr bool KAHAN = sizeof(T) == 4;
    int mx, my, mz;
    long N;
    dasha_params_c P;
    cudaStream_t st;
    // device memory
    void* pool = nullptr;
    T *X[8], *S[8], *A[8], *K[8], *C[8];
    T *cur[2][3], *E[2][3], *Hh[2][3];
    T* tab = nullptr;            // 1-D tables in T
    double* dtab = nullptr;      // 1-D tables in FP64
    double* red = nullptr;       // reduction scratch
    double* cfltab = nullptr;    // CFL rate tables: ich[mx+my+mz], vv[..], ih[..]
    int* flag = nullptr;         // blow-up flag
    unsigned long long* rate_bits = nullptr;   // max CFL rate of the state, from the fused tap
    bool rate_ok = false;        // rate_bits belongs to the current state (set by stepon)
    double* hpin = nullptr;      // pinned host scratch
    double* mpd = nullptr;       // the 11 mid-plane output fields (allocated on first use)
    Geo<T> g{};
    // FP64 device pointers for setdt / diagnostics
    const double *xc, *yc, *zc, *dxs, *dys, *dzs, *wx, *wy, *wz;
    std::vector<double> zcoord, coefz[8];
    std::vector<double> rho0h, b0h[3], p0h, j0h[3];
    bool j0_given = false;
    long nred = 0;
    dim3 blk, grd;
    size_t pool_fbytes = 0;      // bytes per field in the pool (256-byte multiple)
    std::string halo_err;        // the last failed ghost-plane exchange

    SlabGeom slab_geom() const override {
        SlabGeom sg;
        sg.mzl = mz; sg.sz = (long)mx * my; sg.elem = sizeof(T); sg.st = st;
        sg.pool = pool; sg.fbytes = pool_fbytes;
        return sg;
    }
    void set_cfl_k0(int k0) override { g.kcfl0 = k0; }
    // a z-slab with a neighbour: its ghost planes are copies (a lone slab's are the walls)
    bool cut() const { return halo && (halo->geo.lower() || halo->geo.upper()); }
    // z-slab contexts: refresh the ghost planes of fields f that a later launch reads at
    // z-neighbours (a no-op on a whole-grid context)
    void hx(T* const* f, int nf) {
        if (!halo) return;
        void* v[16];
        for (int q = 0; q < nf; ++q) v[q] = f[q];
        if (!halo->exchange(v, nf) && !launch_err) {
            halo_err = "halo exchange: " + halo->err;
            launch_err = halo_err.c_str();
        }
    }

    ~Engine() override {
        xbuf_free();
        if (pool) cudaFree(pool);
        if (tab) cudaFree(tab);
        if (dtab) cudaFree(dtab);
        if (red) cudaFree(red);
        if (cfltab) cudaFree(cfltab);
        if (flag) cudaFree(flag);
        if (rate_bits) cudaFree(rate_bits);
        if (hpin) cudaFreeHost(hpin);
        if (mpd) cudaFree(mpd);
    }

    Status init(int mx_, int my_, int mz_, const dasha_params_c& p, cudaStream_t st_, const HostTables& H) {
        mx = mx_; my = my_; mz = mz_; N = (long)mx * my * mz; P = p; st = st_;
        int nfield = 8 * 4 + (KAHAN ? 8 : 0) + 18;
        size_t fbytes = ((size_t)N * sizeof(T) + 255) & ~(size_t)255;
        size_t freeb = 0, totb = 0;
        DASHA_CK(cudaMemGetInfo(&freeb, &totb));
        if ((double)fbytes * nfield > 0.97 * (double)freeb)
            return Status::err(DASHA_E_NOMEM, "grid needs " + std::to_string((double)fbytes * nfield / 1e9) +
                                                  " GB of device memory, " + std::to_string(freeb / 1e9) + " GB free");
        pool_fbytes = fbytes;
        cudaError_t e = cudaMalloc(&pool, fbytes * nfield);
        if (e != cudaSuccess) { pool = nullptr; cudaGetLastError(); return Status::err(DASHA_E_NOMEM, "cudaMalloc of the field pool failed"); }
        char* q = (char*)pool;
        auto take = [&]() { T* r = (T*)q; q += fbytes; return r; };
        for (int m = 0; m < 8; ++m) X[m] = take();
        for (int m = 0; m < 8; ++m) S[m] = take();
        for (int m = 0; m < 8; ++m) A[m] = take();
        for (int m = 0; m < 8; ++m) K[m] = take();
        for (int m = 0; m < 8; ++m) C[m] = KAHAN ? take() : nullptr;
        for (int b = 0; b < 2; ++b) for (int m = 0; m < 3; ++m) cur[b][m] = take();
        for (int b = 0; b < 2; ++b) for (int m = 0; m < 3; ++m) E[b][m] = take();
        for (int b = 0; b < 2; ++b) for (int m = 0; m < 3; ++m) Hh[b][m] = take();
        DASHA_CK(cudaMemsetAsync(pool, 0, fbytes * nfield, st));

        // T tables: per axis 8 coefficients + wp + wm, plus cbx
        int nx[3] = {mx, my, mz};
        long ntab = 0;
        for (int d = 0; d < 3; ++d) ntab += 11L * nx[d];
        ntab += mx;
        std::vector<T> ht(ntab);
        long off[3][11], offcb;
        long o = 0;
        for (int d = 0; d < 3; ++d)
            for (int q2 = 0; q2 < 11; ++q2) {
                off[d][q2] = o;
                const std::vector<double>& src =
                    q2 < 8 ? H.coef[d][q2] : (q2 == 8 ? H.wp[d] : (q2 == 9 ? H.wm[d] : H.coord[d]));
                for (int i = 0; i < nx[d]; ++i) ht[o + i] = T(src[i]);
                o += nx[d];
            }
        offcb = o;
        for (int i = 0; i < mx; ++i) ht[o + i] = T(H.cbx[i]);
        DASHA_CK(cudaMalloc(&tab, sizeof(T) * ntab));
        DASHA_CK(cudaMemcpy(tab, ht.data(), sizeof(T) * ntab, cudaMemcpyHostToDevice));
        const T* t = tab;
        g.mx = mx; g.my = my; g.mz = mz; g.sy = mx; g.sz = (long)mx * my;
        const T** c1[3][4] = {{&g.a1x, &g.b1x, &g.c1x, &g.d1x}, {&g.a1y, &g.b1y, &g.c1y, &g.d1y}, {&g.a1z, &g.b1z, &g.c1z, &g.d1z}};
        const T** c2[3][4] = {{&g.a2x, &g.b2x, &g.c2x, &g.d2x}, {&g.a2y, &g.b2y, &g.c2y, &g.d2y}, {&g.a2z, &g.b2z, &g.c2z, &g.d2z}};
        const T** w2[3][2] = {{&g.wpx, &g.wmx}, {&g.wpy, &g.wmy}, {&g.wpz, &g.wmz}};
        for (int d = 0; d < 3; ++d) {
            for (int q2 = 0; q2 < 4; ++q2) { *c1[d][q2] = t + off[d][q2]; *c2[d][q2] = t + off[d][4 + q2]; }
            *w2[d][0] = t + off[d][8]; *w2[d][1] = t + off[d][9];
        }
        g.cbx = t + offcb;
        g.xc = t + off[0][10]; g.yc = t + off[1][10]; g.zc = t + off[2][10];
        g.eta = T(p.eta); g.di = T(p.di); g.gamma = T(p.gamma); g.mu = T(p.mu); g.drho = T(p.drho); g.dp = T(p.dp);
        g.hall = p.hall; g.viscos = p.viscos && p.mu != 0.0; g.diffu = p.diffu && (p.drho != 0.0 || p.dp != 0.0);

        // FP64 tables: coords(3), spacing(3), weights(3), equilibrium profiles (16 x mz)
        long nd = 0;
        for (int d = 0; d < 3; ++d) nd += 3L * nx[d];
        nd += 16L * mz;
        std::vector<double> hd(nd, 0.0);
        long od[3][3];
        o = 0;
        for (int d = 0; d < 3; ++d)
            for (int q2 = 0; q2 < 3; ++q2) {
                od[d][q2] = o;
                const std::vector<double>& src = q2 == 0 ? H.coord[d] : (q2 == 1 ? H.spacing[d] : H.weight[d]);
                for (int i = 0; i < nx[d]; ++i) hd[o + i] = src[i];
                o += nx[d];
            }
        long oeq = o;
        DASHA_CK(cudaMalloc(&dtab, sizeof(double) * nd));
        DASHA_CK(cudaMemcpy(dtab, hd.data(), sizeof(double) * nd, cudaMemcpyHostToDevice));
        xc = dtab + od[0][0]; yc = dtab + od[1][0]; zc = dtab + od[2][0];
        dxs = dtab + od[0][1]; dys = dtab + od[1][1]; dzs = dtab + od[2][1];
        wx = dtab + od[0][2]; wy = dtab + od[1][2]; wz = dtab + od[2][2];
        double* eqp = dtab + oeq;
        g.rho0 = eqp; g.bx0 = eqp + mz; g.by0 = eqp + 2 * mz; g.bz0 = eqp + 3 * mz; g.p0 = eqp + 4 * mz;
        g.dzp0 = eqp + 5 * mz; g.d2rho0 = eqp + 6 * mz; g.d2p0 = eqp + 7 * mz;
        g.rsx = eqp + 8 * mz; g.rsy = eqp + 9 * mz; g.rsz = eqp + 10 * mz;
        g.j0x = eqp + 11 * mz; g.j0y = eqp + 12 * mz; g.j0z = eqp + 13 * mz;
        g.dzp0r = eqp + 14 * mz;
        zcoord = H.coord[2];
        for (int q2 = 0; q2 < 8; ++q2) coefz[q2] = H.coef[2][q2];

        {   // CFL rate tables (setdt): 1/(cfl |h|), (eta+mu)/(2 h^2), 1/|h| per axis
            long nt = (long)mx + my + mz;
            std::vector<double> ct(3 * nt);
            long o2 = 0;
            for (int d = 0; d < 3; ++d)
                for (int i2 = 0; i2 < nx[d]; ++i2, ++o2) {
                    double h = H.spacing[d][i2];
                    ct[o2] = 1.0 / (p.cfl * std::fabs(h));
                    ct[nt + o2] = (p.eta + p.mu) / h / 2.0 / h;
                    ct[2 * nt + o2] = 1.0 / std::fabs(h);
                }
            DASHA_CK(cudaMalloc(&cfltab, sizeof(double) * 3 * nt));
            DASHA_CK(cudaMemcpy(cfltab, ct.data(), sizeof(double) * 3 * nt, cudaMemcpyHostToDevice));
        }
        nred = 2L * my * mz + my + 6L * mz + 64;
        DASHA_CK(cudaMalloc(&red, sizeof(double) * (nred + 16)));
        DASHA_CK(cudaMalloc(&flag, sizeof(int)));
        DASHA_CK(cudaMalloc(&rate_bits, sizeof(unsigned long long)));
        DASHA_CK(cudaMemsetAsync(flag, 0, sizeof(int), st));
        DASHA_CK(cudaMallocHost(&hpin, sizeof(double) * 16));

        blk = dim3(std::min(128, ((mx + 31) / 32) * 32));
        grd = dim3((mx + blk.x - 1) / blk.x, my, mz);
        DASHA_CK(zs_attr());
        DASHA_CK(cudaStreamSynchronize(st));
        return Status::ok();
    }

    // 4th-order z-derivative of a profile at interior rows (zero on the wall rows)
    std::vector<double> zderiv(const std::vector<double>& f, int order) const {
        std::vector<double> out(mz, 0.0);
        int base = order == 1 ? 0 : 4;
        for (int k = 2; k <= mz - 3; ++k)
            out[k] = coefz[base][k] * (f[k + 1] - f[k]) + coefz[base + 1][k] * (f[k] - f[k - 1]) +
                     coefz[base + 2][k] * (f[k + 2] - f[k]) + coefz[base + 3][k] * (f[k] - f[k - 2]);
        return out;
    }

    Status upload_eq() {
        rate_ok = false;   // the CFL rate is of the totals: a new equilibrium invalidates it
        std::vector<double> h(16L * mz, 0.0);
        for (int k = 0; k < mz; ++k) {
            h[k] = rho0h[k]; h[mz + k] = b0h[0][k]; h[2 * mz + k] = b0h[1][k]; h[3 * mz + k] = b0h[2][k];
            h[4 * mz + k] = p0h[k];
        }
        std::vector<double> dzp0 = zderiv(p0h, 1), d2r = zderiv(rho0h, 2), d2p = zderiv(p0h, 2);
        std::vector<double> jx(mz, 0.0), jy(mz, 0.0), jz(mz, 0.0);
        if (P.j0_mode == 1) {
            if (j0_given) { jx = j0h[0]; jy = j0h[1]; jz = j0h[2]; }
            else {   // J0 = curl B0(z) = (-dBy0/dz, dBx0/dz, 0)
                std::vector<double> dbx = zderiv(b0h[0], 1), dby = zderiv(b0h[1], 1);
                for (int k = 0; k < mz; ++k) { jx[k] = -dby[k]; jy[k] = dbx[k]; }
            }
        }
        for (int k = 0; k < mz; ++k) {
            h[5 * mz + k] = dzp0[k]; h[6 * mz + k] = d2r[k]; h[7 * mz + k] = d2p[k];
            // xresd: momentum RHS of the pure equilibrium (initia t3dsdsc.f:816-834); the flux
            // divergence and J1 vanish there, leaving J0 x B0 (zero in LITERAL mode)
            double rx = 0., ry = 0., rz = 0.;
            if (P.j0_mode == 1 && k >= 2 && k <= mz - 3) {
                double b1 = b0h[0][k], b2 = b0h[1][k], b3 = b0h[2][k];
                rx = jy[k] * b3 - jz[k] * b2;
                ry = jz[k] * b1 - jx[k] * b3;
                rz = jx[k] * b2 - jy[k] * b1;
            }
            h[8 * mz + k] = rx; h[9 * mz + k] = ry; h[10 * mz + k] = rz;
            h[11 * mz + k] = jx[k]; h[12 * mz + k] = jy[k]; h[13 * mz + k] = jz[k];
            h[14 * mz + k] = dzp0[k] / rho0h[k];
        }
        DASHA_CK(cudaMemcpyAsync((void*)g.rho0, h.data(), sizeof(double) * 16 * mz, cudaMemcpyHostToDevice, st));
        DASHA_CK(cudaStreamSynchronize(st));
        return Status::ok();
    }

    Status set_equilibrium(const double* rho0, const double* b0, const double* p0, const double*) override {
        rho0h.assign(rho0, rho0 + mz);
        for (int m = 0; m < 3; ++m) b0h[m].assign(b0 + m * mz, b0 + (m + 1) * mz);
        p0h.assign(p0, p0 + mz);
        return upload_eq();
    }
    Status set_j0(const double* j0) override {
        for (int m = 0; m < 3; ++m) j0h[m].assign(j0 + m * mz, j0 + (m + 1) * mz);
        j0_given = true;
        return upload_eq();
    }

    // ---- host array transfer through a FP64 staging buffer, one field at a time ----
    // ---- host <-> device transfer of fields in the caller's Fortran halo layout ----
    // Chunks of whole z planes (compact mx x my x nk doubles) move through two pinned host
    // buffers and two device buffers: host threads gather (scatter) the interior rows of the
    // caller's array into (out of) one pinned buffer while the other's DMA and conversion
    // kernel run.  Only interior entries are written back, so the caller's halo entries keep
    // their values.
    double* xh[2] = {nullptr, nullptr};   // pinned host chunk buffers
    double* xd[2] = {nullptr, nullptr};   // device chunk buffers
    cudaEvent_t xev[2] = {nullptr, nullptr};
    int xnk = 0;                          // z planes per chunk
    Status xbuf() {
        if (xh[0]) return Status::ok();
        const size_t pb = sizeof(double) * (size_t)mx * my;
        xnk = (int)std::max<size_t>(1, std::min<size_t>((size_t)mz, (size_t(64) << 20) / pb));
        for (int b = 0; b < 2; ++b) {
            DASHA_CK(cudaMallocHost(&xh[b], pb * xnk));
            DASHA_CK(cudaMalloc(&xd[b], pb * xnk));
            DASHA_CK(cudaEventCreateWithFlags(&xev[b], cudaEventDisableTiming));
        }
        return Status::ok();
    }
    void xbuf_free() {
        for (int b = 0; b < 2; ++b) {
            if (xh[b]) cudaFreeHost(xh[b]);
            if (xd[b]) cudaFree(xd[b]);
            if (xev[b]) cudaEventDestroy(xev[b]);
            xh[b] = xd[b] = nullptr;
            xev[b] = nullptr;
        }
    }
    // f(r0, r1) over rows [0, n), split across the host thread pool
    template <class F>
    static void par_rows(long n, F f) { HostPool::get().run(n, f); }
    // Chunked host transfers.  z-plane chunks of one field move through the two pinned host
    // buffers and the two device buffers, so that the host work on one chunk overlaps the DMA
    // and the conversion kernel of the other.  The host work is the caller's: fill(m, k0, k1,
    // rows) writes field m on planes k0..k1-1 as (k1-k0)*my rows of mx values (x fastest)
    // before they go to the device; take(m, k0, k1, rows) reads them after they arrive.  A
    // false return ends the transfer with DASHA_E_INVALID; the fields moved before it stay.
    Status stream_in(T* const* dst, int nf, bool sub_eq, const ChunkIn& fill) {
        Status s = xbuf();
        if (s.code) return s;
        int q = 0;
        for (int m = 0; m < nf; ++m) {
            const double* prof = sub_eq ? eq_profile(g, m) : nullptr;
            for (int k0 = 0; k0 < mz; k0 += xnk, ++q) {
                const int k1 = std::min(mz, k0 + xnk), b = q & 1;
                DASHA_CK(cudaEventSynchronize(xev[b]));        // the DMA out of xh[b] is done
                if (!fill(m, k0, k1, xh[b])) {
                    DASHA_CK(cudaStreamSynchronize(st));
                    return Status::err(DASHA_E_INVALID, "the host side of the transfer failed");
                }
                DASHA_CK(cudaMemcpyAsync(xd[b], xh[b], sizeof(double) * (size_t)mx * my * (k1 - k0), cudaMemcpyHostToDevice, st));
                DASHA_CK(cudaEventRecord(xev[b], st));
                k_import_chunk<T><<<dim3((mx + blk.x - 1) / blk.x, my, k1 - k0), blk, 0, st>>>(mx, my, k0, xd[b], prof, dst[m]);
                DASHA_CK(cudaGetLastError());
            }
        }
        DASHA_CK(cudaStreamSynchronize(st));
        return Status::ok();
    }

    Status stream_out(T* const* src, int nf, bool add_eq, T* const* comp, const ChunkOut& take) {
        Status s = xbuf();
        if (s.code) return s;
        struct Pend { int m, k0, k1, b; };
        Pend prev{-1, 0, 0, 0};
        bool ok = true;
        auto drain = [&](const Pend& c) -> Status {
            DASHA_CK(cudaEventSynchronize(xev[c.b]));       // its D2H has landed
            ok = take(c.m, c.k0, c.k1, xh[c.b]);
            return Status::ok();
        };
        int q = 0;
        for (int m = 0; m < nf && ok; ++m) {
            const double* prof = add_eq ? eq_profile(g, m) : nullptr;
            for (int k0 = 0; k0 < mz && ok; k0 += xnk, ++q) {
                const int k1 = std::min(mz, k0 + xnk), b = q & 1;
                k_export_chunk<T><<<dim3((mx + blk.x - 1) / blk.x, my, k1 - k0), blk, 0, st>>>(
                    mx, my, k0, src[m], comp ? comp[m] : nullptr, prof, xd[b]);
                DASHA_CK(cudaGetLastError());
                DASHA_CK(cudaMemcpyAsync(xh[b], xd[b], sizeof(double) * (size_t)mx * my * (k1 - k0), cudaMemcpyDeviceToHost, st));
                DASHA_CK(cudaEventRecord(xev[b], st));
                if (prev.m >= 0) {                             // the previous chunk meanwhile
                    s = drain(prev);
                    if (s.code) return s;
                }
                prev = {m, k0, k1, b};
            }
        }
        if (ok && prev.m >= 0) {
            s = drain(prev);
            if (s.code) return s;
        }
        DASHA_CK(cudaStreamSynchronize(st));
        if (!ok) return Status::err(DASHA_E_INVALID, "the host side of the transfer failed");
        return Status::ok();
    }

    // The same with the caller's array in the reference layout: node (i, j, k) of field m at
    // (i+2) + ld1 (j + ld2 ((k+2) + (mz+4) m)); rows are gathered (scattered) by host threads.
    ChunkIn gather(const double* host, long ld1, long ld2) const {
        const size_t fld = (size_t)ld1 * ld2 * (mz + 4);
        const int mx_ = mx, my_ = my;
        return [=](int m, int k0, int k1, double* rows) {
            const double* srcp = host + fld * m;
            par_rows((long)(k1 - k0) * my_, [&](long r0, long r1) {
                for (long r = r0; r < r1; ++r) {
                    const long kk = k0 + r / my_, j = r % my_;
                    std::memcpy(rows + r * mx_, srcp + 2 + ld1 * (j + ld2 * (kk + 2)), sizeof(double) * mx_);
                }
            });
            return true;
        };
    }
    ChunkOut scatter(double* host, long ld1, long ld2) const {
        const size_t fld = (size_t)ld1 * ld2 * (mz + 4);
        const int mx_ = mx, my_ = my;
        return [=](int m, int k0, int k1, const double* rows) {
            double* dstp = host + fld * m;
            par_rows((long)(k1 - k0) * my_, [&](long r0, long r1) {
                for (long r = r0; r < r1; ++r) {
                    const long kk = k0 + r / my_, j = r % my_;
                    std::memcpy(dstp + 2 + ld1 * (j + ld2 * (kk + 2)), rows + r * mx_, sizeof(double) * mx_);
                }
            });
            return true;
        };
    }
    Status transfer_in(const double* host, long ld1, long ld2, T* const* dst, int nf, bool sub_eq) {
        return stream_in(dst, nf, sub_eq, gather(host, ld1, ld2));
    }
    Status transfer_out(double* host, long ld1, long ld2, T* const* src, int nf, bool add_eq,
                        T* const* comp = nullptr) {
        return stream_out(src, nf, add_eq, comp, scatter(host, ld1, ld2));
    }

    Status state_in(const ChunkIn& fill) override {
        rate_ok = false;
        Status s = stream_in(X, 8, true, fill);
        if (s.code) return s;
        if (KAHAN) for (int m = 0; m < 8; ++m) DASHA_CK(cudaMemsetAsync(C[m], 0, sizeof(T) * N, st));
        DASHA_CK(cudaMemsetAsync(flag, 0, sizeof(int), st));
        DASHA_CK(cudaStreamSynchronize(st));
        return Status::ok();
    }
    Status state_out(const ChunkOut& take) override { return stream_out(X, 8, true, KAHAN ? C : nullptr, take); }

    int raw_fields() const override { return KAHAN ? 16 : 8; }
    size_t raw_elem() const override { return sizeof(T); }
    Status raw_out(const std::function<bool(const void*, size_t)>& take) override {
        Status s = xbuf();
        if (s.code) return s;
        const size_t cap = sizeof(double) * (size_t)mx * my * xnk, total = sizeof(T) * (size_t)N;
        for (int f = 0; f < raw_fields(); ++f) {
            const char* src = reinterpret_cast<const char*>(f < 8 ? X[f] : C[f - 8]);
            for (size_t o = 0; o < total; o += cap) {
                const size_t n = std::min(cap, total - o);
                DASHA_CK(cudaMemcpyAsync(xh[0], src + o, n, cudaMemcpyDeviceToHost, st));
                DASHA_CK(cudaStreamSynchronize(st));
                if (!take(xh[0], n)) return Status::err(DASHA_E_INVALID, "the host side of the transfer failed");
            }
        }
        return Status::ok();
    }
    Status raw_in(const std::function<bool(void*, size_t)>& give) override {
        Status s = xbuf();
        if (s.code) return s;
        const size_t cap = sizeof(double) * (size_t)mx * my * xnk, total = sizeof(T) * (size_t)N;
        // into S (and A for the FP32 compensations), spare between steps, then swapped in
        for (int f = 0; f < raw_fields(); ++f) {
            char* dst = reinterpret_cast<char*>(f < 8 ? S[f] : A[f - 8]);
            for (size_t o = 0; o < total; o += cap) {
                const size_t n = std::min(cap, total - o);
                if (!give(xh[0], n)) return Status::err(DASHA_E_INVALID, "the host side of the transfer failed");
                DASHA_CK(cudaMemcpyAsync(dst + o, xh[0], n, cudaMemcpyHostToDevice, st));
                DASHA_CK(cudaStreamSynchronize(st));
            }
        }
        for (int m = 0; m < 8; ++m) {
            std::swap(X[m], S[m]);
            if (KAHAN) std::swap(C[m], A[m]);
        }
        DASHA_CK(cudaMemsetAsync(flag, 0, sizeof(int), st));
        DASHA_CK(cudaStreamSynchronize(st));
        rate_ok = false;
        return Status::ok();
    }
    Status set_state(const double* x, long ld1, long ld2) override { return state_in(gather(x, ld1, ld2)); }
    Status get_state(double* x, long ld1, long ld2) override { return state_out(scatter(x, ld1, ld2)); }

    // ---- the RHS chain (right, t3dsdsc.f:1297-1673) ----
    static F8<T> f8(T* const* p) { F8<T> r; for (int m = 0; m < 8; ++m) r.f[m] = p[m]; return r; }
    static F3<T> f3(T* const* p) { F3<T> r; for (int m = 0; m < 3; ++m) r.f[m] = p[m]; return r; }

    // ---- z-marching launches ----
    static constexpr int TX = 32, TY = 8;
    int zchunk(int gxy, int minlen) const {
        int nch = (4 * 148 * 8 + gxy - 1) / gxy;
        nch = std::max(1, std::min(nch, mz / minlen));
        return (mz + nch - 1) / nch;
    }
    // radius-2 ring kernels (k_zst2): 32 x 8 columns per CTA
    static constexpr int ZTX = 32;
    // k_zpv tiling: a warp covers 32*ZVX x nodes (float pairs in FP32), a thread RY
    // consecutive rows, TYH warps per CTA, D planes in flight.  Measured best on the
    // 1024x512x1024 FP32 and 512x256x512 FP64 steps: FP32 64x8 tiles of 256 threads (one row
    // each, 3 planes ahead); FP64 32x8 tiles of 128 threads (two rows each, 2 planes ahead).
    static constexpr int ZVX = sizeof(T) == 4 ? 2 : 1;
    template <int NF>
    struct ZC {
        static constexpr int TYH = sizeof(T) == 4 ? 8 : 4;
        static constexpr int RY = sizeof(T) == 4 ? 1 : 2;
        static constexpr int D = sizeof(T) == 4 ? 3 : 2;
    };
    template <int NF>
    using ZVc = ZV<T, NF, ZVX, ZC<NF>::TYH, ZC<NF>::RY, ZC<NF>::D>;
    template <int NF, unsigned KINDS, class Epi, int MODE>
    static constexpr auto zpv_fn() { return k_zpv<T, NF, KINDS, ZVX, ZC<NF>::TYH, ZC<NF>::RY, ZC<NF>::D, Epi, MODE>; }
#ifndef DASHA_NO_TMA
    template <int NF, unsigned KINDS, class Epi, int MODE>
    static constexpr auto zpv_tma_fn() { return k_zpv_tma<T, NF, KINDS, ZVX, ZC<NF>::TYH, ZC<NF>::RY, ZC<NF>::D, Epi, MODE>; }
    // the source fields of a pass as tensor maps, boxes of one ring plane (RS x NR x 1)
    template <int NF>
    bool zpv_maps(const SrcFields<T, NF>& src, ZpMaps& m) {
        using Z = ZVc<NF>;
        EncodeTiledFn enc = encode_tiled();
        if (!enc) return false;
        const cuuint64_t dims[3] = {(cuuint64_t)mx, (cuuint64_t)my, (cuuint64_t)mz};
        const cuuint64_t strides[2] = {(cuuint64_t)g.sy * sizeof(T), (cuuint64_t)g.sz * sizeof(T)};
        const cuuint32_t box[3] = {(cuuint32_t)Z::RS, (cuuint32_t)Z::NR, 1u};
        const cuuint32_t estr[3] = {1u, 1u, 1u};
        const CUtensorMapDataType dt = sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
        for (int q = 0; q < NF; ++q)
            if (enc(&m.m[q], dt, 3u, const_cast<T*>(src.f[q]), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                    CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
                return false;
        return true;
    }
#endif
    // Ring loads by TMA where they measured faster on B200 (1024x512x1024 FP32, 512x256x512 FP64,
    // bitwise the same states): every FP64 pass (4-9 % faster) and the FP64 hydro RHS (13 %); in
    // FP32 the passes of 4 and 6 fields (the summed E/Hall pass 18 %, filter pass 1 14 %) and the
    // hydro RHS (2 %), while the 3-field passes stay on cp.async (TMA 10 % slower there)
#if defined(DASHA_TMA_ALL)
    template <int NF>
    static constexpr bool zp_tma() { return true; }                  // measurement build: every pass
#elif !defined(DASHA_NO_TMA)
    template <int NF>
    static constexpr bool zp_tma() { return sizeof(T) == 8 || NF >= 4; }
#else
    template <int NF>
    static constexpr bool zp_tma() { return false; }
#endif
    // one smoothing pass of NF fields: src -> epi
    template <int NF, unsigned KINDS, int MODE = 0, class Epi>
    void zp(const char* tag, double bytes, const SrcFields<T, NF>& src, const Epi& epi) {
        using Z = ZVc<NF>;
        dim3 gg((mx + Z::TX - 1) / Z::TX, (my + Z::TY - 1) / Z::TY, 1);
        int ch = zchunk(gg.x * gg.y, 16);
        gg.z = (mz + ch - 1) / ch;
#ifndef DASHA_NO_TMA
        if constexpr (zp_tma<NF>()) {
            ZpMaps maps;
            if (!zpv_maps<NF>(src, maps)) launch_err = "cuTensorMapEncodeTiled failed for a smoothing pass";
            DASHA_LAUNCH(tag, bytes, (zpv_tma_fn<NF, KINDS, Epi, MODE>()<<<gg, 32 * ZC<NF>::TYH, Z::smem_tma(), st>>>(g, src, epi, ch, maps)));
        } else
#endif
        {
            DASHA_LAUNCH(tag, bytes, (zpv_fn<NF, KINDS, Epi, MODE>()<<<gg, 32 * ZC<NF>::TYH, Z::smem(), st>>>(g, src, epi, ch)));
        }
    }
    template <int NF, unsigned KINDS, class Epi, int MODE = 0>
    static cudaError_t zp_attr1() {
#ifndef DASHA_NO_TMA
        if constexpr (zp_tma<NF>())
            return cudaFuncSetAttribute(zpv_tma_fn<NF, KINDS, Epi, MODE>(), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)ZVc<NF>::smem_tma());
#endif
        return cudaFuncSetAttribute(zpv_fn<NF, KINDS, Epi, MODE>(), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)ZVc<NF>::smem());
    }
    // k_zpv2 (two passes in one launch): tile 32*ZVX x 8, one row per warp plus two halo-row
    // warps, D planes in flight
    // (measurement builds may set the tile height and depth: -DDASHA_ZP2_TY=.. -DDASHA_ZP2_D=..)
    template <int NF>
    struct ZC2 {
#ifdef DASHA_ZP2_TY
        static constexpr int TY = DASHA_ZP2_TY;
#else
        static constexpr int TY = 8;
#endif
#ifdef DASHA_ZP2_D
        static constexpr int D = DASHA_ZP2_D;
#else
        static constexpr int D = sizeof(T) == 4 ? 3 : 2;
#endif
    };
    template <int NF>
    using ZV2c = ZV2<T, NF, ZVX, ZC2<NF>::TY, ZC2<NF>::D>;
    template <int NF, unsigned KINDS, class Epi>
    static constexpr auto zpv2_fn() { return k_zpv2<T, NF, KINDS, ZVX, ZC2<NF>::TY, ZC2<NF>::D, Epi>; }
    // two smoothing passes of NF fields: src -> epi (src must not alias the epilogue's outputs)
    template <int NF, unsigned KINDS, class Epi>
    void zp2(const char* tag, double bytes, const SrcFields<T, NF>& src, const Epi& epi) {
        using Z = ZV2c<NF>;
        dim3 gg((mx + Z::TX - 1) / Z::TX, (my + ZC2<NF>::TY - 1) / ZC2<NF>::TY, 1);
        int ch = zchunk(gg.x * gg.y, 16);
        gg.z = (mz + ch - 1) / ch;
        DASHA_LAUNCH(tag, bytes, (zpv2_fn<NF, KINDS, Epi>()<<<gg, 32 * Z::NW, Z::smem(), st>>>(g, src, epi, ch)));
    }
    template <int NF, unsigned KINDS, class Epi>
    static cudaError_t zp2_attr1() {
        return cudaFuncSetAttribute(zpv2_fn<NF, KINDS, Epi>(), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)ZV2c<NF>::smem());
    }
    // k_zcurl: tile 32*ZVX x 8, one row per warp, 2 planes in flight beyond c+2
    using ZC3c = ZC3<T, ZVX, 8, 2>;
    template <int SIGN>
    void zcurl(const char* tag, const SrcFields<T, 3>& src, F3<T> out) {
        dim3 gg((mx + ZC3c::TX - 1) / ZC3c::TX, (my + 7) / 8, 1);
        int ch = zchunk(gg.x * gg.y, 16);
        gg.z = (mz + ch - 1) / ch;
        DASHA_LAUNCH(tag, 6.0 * N * sizeof(T), (k_zcurl<T, ZVX, 8, 2, SIGN><<<gg, 256, ZC3c::smem(), st>>>(g, src, out, ch)));
    }
    // k_zhydro: one node per thread, tile 32 x 4, 1 plane in flight beyond c+2, 4 (FP32) or 3
    // (FP64) CTAs per SM.  Measured (hydro ms per step, FP32 1024x512x1024 / FP64 512x256x512):
    // float pairs, 8 rows, 1 CTA/SM 57.5 / -; pairs capped at 2 CTAs/SM (spills) 73.9 / -; one
    // node per thread, 4 rows, 4 CTAs/SM 55.3 / -; 8 rows, 1 CTA/SM - / 16.6; 4 rows, 3 CTAs/SM
    // 60.8 (pairs) / 12.8; 8 rows capped at 3 CTAs (spills) 66.5 / -
    static constexpr int ZH_VX = 1, ZH_TY = 4, ZH_MINB = sizeof(T) == 4 ? 4 : 3;
    using ZHc = ZH<T, ZH_VX, ZH_TY, 1>;
    using ZEHc = ZEH<T, ZVX, 8, 2>;   // k_zeh: tile 32*ZVX x 8, 2 planes in flight beyond c+2
    using St3 = VStore<T, 3, ZVX>;
    using St4 = VStore<T, 4, ZVX>;
    using Acc3 = VAcc<T, 3, ZVX>;
    using RK4 = VRK<T, 4, ZVX, KAHAN>;
    cudaError_t zs_attr() {
        cudaError_t e;
        if ((e = zp_attr1<3, 0u, St3>())) return e;
        if ((e = zp_attr1<3, KIND_H, St3>())) return e;
        if ((e = zp_attr1<3, KIND_H, Acc3>())) return e;
        if ((e = zp_attr1<6, KIND_EH, VSum<T, 3, ZVX>>())) return e;
        if ((e = zp_attr1<4, 0u, St4>())) return e;
        if ((e = zp_attr1<4, KIND_B4, St4>())) return e;
        if ((e = zp_attr1<4, 0u, RK4>())) return e;
        if ((e = zp_attr1<4, KIND_B4, RK4>())) return e;
        if ((e = zp_attr1<4, KIND_B4, WithCfl<St4, T, ZVX>>())) return e;
        if ((e = zp2_attr1<3, KIND_H, St3>())) return e;
        if constexpr (KAHAN) {
            if ((e = zp_attr1<4, 0u, VStore<T, 2, ZVX>, 1>())) return e;
            if ((e = zp_attr1<4, KIND_P45, VStore<T, 2, ZVX>, 1>())) return e;
            if ((e = zp_attr1<4, KIND_P67, VStore<T, 2, ZVX>, 1>())) return e;
            if ((e = zp_attr1<4, 0u, VKF<T, 4, ZVX>, 2>())) return e;
            if ((e = zp_attr1<4, KIND_B4, VKF<T, 4, ZVX>, 2>())) return e;
            if ((e = zp_attr1<4, KIND_B4, WithCfl<VKF<T, 4, ZVX>, T, ZVX>, 2>())) return e;
        }
        if ((e = cudaFuncSetAttribute(k_zst2<T, 5, ZTX, 8, HMINB, OpHydro<T>>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)ZS2<T, 5, ZTX, 8>::smem(true))))
            return e;
        if ((e = cudaFuncSetAttribute(k_zeh<T, ZVX, 8, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)ZEHc::smem())))
            return e;
        if ((e = cudaFuncSetAttribute(k_zhydro<T, ZH_VX, ZH_TY, 1, ZH_MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)ZHc::smem())))
            return e;
#ifndef DASHA_NO_TMA
        if ((e = cudaFuncSetAttribute(k_zhydro_tma<T, ZH_VX, ZH_TY, 1, ZH_MINB>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ZHc::smem_tma())))
            return e;
#endif
        if ((e = cudaFuncSetAttribute(k_zcurl<T, ZVX, 8, 2, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)ZC3c::smem())))
            return e;
        return cudaFuncSetAttribute(k_zcurl<T, ZVX, 8, 2, -1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)ZC3c::smem());
    }
    static constexpr int HMINB = sizeof(T) == 4 ? 2 : 1;   // CTAs per SM asked of the register allocator
    static SrcFields<T, 3> src3(T* const* p) { SrcFields<T, 3> s; for (int q = 0; q < 3; ++q) s.f[q] = p[q]; return s; }
    static SrcFields<T, 8> src8(T* const* p) { SrcFields<T, 8> s; for (int q = 0; q < 8; ++q) s.f[q] = p[q]; return s; }
    static St3 st3(T* const* p) { St3 s; for (int q = 0; q < 3; ++q) s.f[q] = p[q]; return s; }
    static constexpr unsigned KIND_H = 1u | (1u << 2) | (1u << 4);                 // 1/8 for 3 fields
    static constexpr unsigned KIND_B4 = 2u | (2u << 2) | (2u << 4);                 // fields 4..7: B1 B2 B3 p
    static constexpr unsigned KIND_P45 = 2u | (2u << 2);                            // field pair (B1, B2)
    static constexpr unsigned KIND_EH = (1u << 6) | (1u << 8) | (1u << 10);         // E (radial) then Hall (1/8)
    static constexpr unsigned KIND_P67 = 2u;                                        // field pair (B3, p)

    // one avrg/avrgtt pass over the 8 state-like fields, as two 4-field launches (rho, m) and
    // (B, p); mk(lo) builds the epilogue of fields lo..lo+3
    template <class MkEpi>
    void pass8(const char* tag, double bytes_per_cell, T* const* in, MkEpi mk) {
        SrcFields<T, 4> a, b;
        for (int q = 0; q < 4; ++q) { a.f[q] = in[q]; b.f[q] = in[4 + q]; }
        zp<4, 0u>(tag, 0.5 * bytes_per_cell * N * sizeof(T), a, mk(0));
        zp<4, KIND_B4>(tag, 0.5 * bytes_per_cell * N * sizeof(T), b, mk(4));
    }
    static St4 st4(T* const* p, int lo) { St4 s; for (int q = 0; q < 4; ++q) s.f[q] = p[lo + q]; return s; }
    // values per field the RK stage epilogue reads and writes (base, acc, x, comp)
    static constexpr double rk_io(int stage) { return stage == 1 ? 3.0 : (stage < 4 ? 4.0 : (KAHAN ? 5.0 : 2.0)); }
    // both xdif avrg passes of the raw RHS k, the second ending in the RK stage update: x =
    // stage state (or the step result at stage 4), base, acc, comp (FP32 Kahan compensation or
    // null)
    // The fused CFL tap (CflTap, mhd_kernels.cuh) reading back the final state f, its maximum
    // into rate_bits (cleared here, on the stream, before the tapped launch)
    CflTap<T> cfl_tap(T* const* f) {
        CflTap<T> c;
        for (int m = 0; m < 8; ++m) c.x.f[m] = f[m];
        const long nt = (long)mx + my + mz;
        c.ich = cfltab; c.vv = cfltab + nt; c.ih = cfltab + 2 * nt;
        c.rho0 = g.rho0; c.bx0 = g.bx0; c.by0 = g.by0; c.bz0 = g.bz0; c.p0 = g.p0;
        c.gamma = P.gamma;
        c.whistler = (P.dt_whistler && P.hall) ? P.di * 3.141592653589793 : 0.0;
        c.mx = mx; c.my = my; c.mz = mz; c.sy = (unsigned)mx; c.sz = (unsigned)((long)mx * my);
        c.out = rate_bits;
        cudaMemsetAsync(rate_bits, 0, sizeof(unsigned long long), st);
        return c;
    }
    template <class E>
    WithCfl<E, T, ZVX> with_cfl(const E& e, T* const* f) {
        WithCfl<E, T, ZVX> w;
        static_cast<E&>(w) = e;
        w.tap = cfl_tap(f);
        w.best = 0.0;
        return w;
    }
    // the tap reads 8 fields back per node: 4 finished by the launch before (DRAM), 4 just
    // stored (L2)
    double tap_bytes() const { return 4.0 * sizeof(T) * N; }

    // both xdif avrg passes of the raw RHS k, the second ending in the RK stage update: x =
    // stage state (or the step result at stage 4), base, acc, comp (FP32 Kahan compensation or
    // null)
    void rk_passes(int stage, double dt, T* const* k, T* const* base, T* const* x, T* const* acc, T* const* comp) {
        static const char* names[4] = {"k_zpv_X_rk1", "k_zpv_X_rk2", "k_zpv_X_rk3", "k_zpv_X_rk4"};
        T* t[8];
        tmp8(t);
        pass8("k_zpv_X", 16.0, k, [&](int lo) { return st4(t, lo); });
        hx(t, 8);
        auto mk = [&](int lo) {
            RK4 er;
            for (int m = 0; m < 4; ++m) {
                er.x[m] = x[lo + m]; er.base[m] = base[lo + m]; er.acc[m] = acc[lo + m];
                er.comp[m] = comp ? comp[lo + m] : nullptr;
            }
            er.stage = stage;
            er.dt = dt;
            return er;
        };
        pass8(names[stage - 1], 8.0 * (1.0 + rk_io(stage)), t, mk);
        if (stage < 4) hx(x, 8);   // the next stage's state
    }

    // avrgtt on the compensated FP32 state (X, C): pass 1 writes its increment of X - C into
    // t, pass 2 adds the two-pass increment to (X, C) in place with a Kahan step
    void filter_compensated(T* const* t, bool tap = false) {
        for (int lo = 0; lo < 8; lo += 2) {   // pass 1 by field pairs: ring (x_a, x_b, comp_a, comp_b)
            SrcFields<T, 4> a;
            VStore<T, 2, ZVX> o;
            for (int q = 0; q < 2; ++q) { a.f[q] = X[lo + q]; a.f[2 + q] = C[lo + q]; o.f[q] = t[lo + q]; }
            const double by = 6.0 * N * sizeof(T);
            if (lo < 4) zp<4, 0u, 1>("k_zpv_F1", by, a, o);
            else if (lo == 4) zp<4, KIND_P45, 1>("k_zpv_F1", by, a, o);
            else zp<4, KIND_P67, 1>("k_zpv_F1", by, a, o);
        }
        hx(t, 8);
        for (int lo = 0; lo < 8; lo += 4) {
            SrcFields<T, 4> d;
            VKF<T, 4, ZVX> e;
            for (int q = 0; q < 4; ++q) { d.f[q] = t[lo + q]; e.x[q] = X[lo + q]; e.comp[q] = C[lo + q]; }
            if (lo == 0) zp<4, 0u, 2>("k_zpv_F2", 20.0 * N * sizeof(T), d, e);
            else if (!tap) zp<4, KIND_B4, 2>("k_zpv_F2", 20.0 * N * sizeof(T), d, e);
            else zp<4, KIND_B4, 2>("k_zpv_F2", 20.0 * N * sizeof(T) + tap_bytes(), d, with_cfl(e, X));
        }
    }

    T** curF = nullptr;   // smoothed current after launch_current
    T** Ef = nullptr;     // total E after launch_rhs_raw

    // n smoothing passes of 3 fields, ping-pong between a and b starting from a; returns the
    // buffer holding the result.  On a z-slab every pass output that a later pass reads has its
    // ghost planes refreshed, the last one too when xlast (a later launch reads it at
    // z-neighbours), and the Hall pairs run as single passes: k_zpv2 forms its first pass on the
    // planes next to the slab ends from the wall rule.  Both give the same values: the fused
    // pair rounds as two single passes.
    // Pass pairs of the Hall chain (constant coefficient 1/8) run fused in k_zpv2.  Measured on
    // B200 (FP32 1024x512x1024 / FP64 512x256x512 step): Hall pairs fused 436.0 / 107.7 ms,
    // nothing fused 442.1 / 108.4; fusing the radial-coefficient chains J and E as well 437.3 /
    // 186.7 with everything; the xdif pair with the RK update 138.4 (FP64), the FP64 filter
    // 114.1: where the coefficient is evaluated per node, or the epilogue is heavy, the doubled
    // per-node work and the lower occupancy of the 320-thread CTA outweigh the saved traffic.
    template <unsigned KINDS>
    T** passes3(const char* tag, T** a, T** b, int n, bool xlast) {
        if constexpr (KINDS == KIND_H) {
            if (!cut()) {
                for (int p = 0; p < n; p += 2) {   // pairs of passes in one k_zpv2 launch, a lone last one by k_zpv
                    T** in = ((p / 2) & 1) ? b : a;
                    T** out = ((p / 2) & 1) ? a : b;
                    if (p + 1 < n) zp2<3, KINDS>(tag, 6.0 * N * sizeof(T), src3(in), st3(out));
                    else zp<3, KINDS>(tag, 6.0 * N * sizeof(T), src3(in), st3(out));
                }
                return (((n + 1) / 2) & 1) ? b : a;
            }
        }
        for (int p = 0; p < n; ++p) {
            T** in = (p & 1) ? b : a;
            T** out = (p & 1) ? a : b;
            zp<3, KINDS>(tag, 6.0 * N * sizeof(T), src3(in), st3(out));
            if (p < n - 1 || xlast) hx(out, 3);
        }
        return (n & 1) ? b : a;
    }

    // smoothed current of state xs (current, t3dsdsc.f:2452-2500): curl, 4 passes
    const char* launch_err = nullptr;   // a launch that could not be set up (reported by stepon)
#ifndef DASHA_NO_TMA
    // the five ring fields of k_zhydro as tensor maps, boxes of one ring plane (RS x NR x 1)
    bool hydro_maps(const HydroIO<T>& io, ZhMaps& m) {
        EncodeTiledFn enc = encode_tiled();
        if (!enc) return false;
        const T* f[5] = {io.m1, io.m2, io.m3, io.dp, io.drho};
        const cuuint64_t dims[3] = {(cuuint64_t)mx, (cuuint64_t)my, (cuuint64_t)mz};
        const cuuint64_t strides[2] = {(cuuint64_t)g.sy * sizeof(T), (cuuint64_t)g.sz * sizeof(T)};
        const cuuint32_t box[3] = {(cuuint32_t)ZHc::RS, (cuuint32_t)ZHc::NR, 1u};
        const cuuint32_t estr[3] = {1u, 1u, 1u};
        const CUtensorMapDataType dt = sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
        for (int q = 0; q < 5; ++q)
            if (enc(&m.m[q], dt, 3u, const_cast<T*>(f[q]), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                    CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
                return false;
        return true;
    }
#endif
    void launch_current(T* const* xs) {
        T* bb[3] = {xs[4], xs[5], xs[6]};
        zcurl<1>("k_curl", src3(bb), f3(cur[0]));
        hx(cur[0], 3);
        curF = passes3<0u>("k_zpv_J", cur[0], cur[1], 4, false);
        if (P.j0_mode == 1) DASHA_LAUNCH("k_add_j0", 6.0 * N * sizeof(T), k_add_j0<T><<<grd, blk, 0, st>>>(g, f3(curF)));
    }

    // E_total and the raw RHS of state xs into K (wall rows applied)
    void launch_rhs_raw(T* const* xs) {
        NvtxRange range("right");
        launch_current(xs);
        T** cother = curF == cur[0] ? cur[1] : cur[0];
        (void)cother;
        // E0 = -v x B + eta J at every node, then avrgE's 4 passes (t3dsdsc.f:1367-1389)
        if (P.hall) {   // E0 and the Hall field in one z-march over the state
            EHIO<T> eh;
            eh.drho = xs[0]; eh.m1 = xs[1]; eh.m2 = xs[2]; eh.m3 = xs[3];
            eh.b1 = xs[4]; eh.b2 = xs[5]; eh.b3 = xs[6]; eh.dp = xs[7];
            eh.j1 = curF[0]; eh.j2 = curF[1]; eh.j3 = curF[2];
            for (int q = 0; q < 3; ++q) { eh.e[q] = E[0][q]; eh.h[q] = Hh[0][q]; }
            dim3 ge((mx + ZEHc::TX - 1) / ZEHc::TX, (my + 7) / 8, 1);
            int che = zchunk(ge.x * ge.y, 16);
            ge.z = (mz + che - 1) / che;
            DASHA_LAUNCH("k_efield_hall", 17.0 * N * sizeof(T), (k_zeh<T, ZVX, 8, 2><<<ge, 256, ZEHc::smem(), st>>>(g, eh, che)));
            hx(Hh[0], 3);
        } else {
            DASHA_LAUNCH("k_efield", 13.0 * N * sizeof(T), k_efield<T><<<grd, blk, 0, st>>>(g, f8(xs), f3(curF), f3(E[0])));
        }
        hx(E[0], 3);
        if (P.hall) {
            // avrgh passes 1-4, avrgE passes 1-3, then one 6-field launch: the 4th E pass and the
            // 5th Hall pass, summed into E (the two chains are independent until that sum)
            T** h = passes3<KIND_H>("k_zpv_H", Hh[0], Hh[1], 4, true);
            T** e3 = passes3<0u>("k_zpv_E", E[0], E[1], 3, true);
            T** eo = e3 == E[0] ? E[1] : E[0];
            SrcFields<T, 6> se;
            VSum<T, 3, ZVX> es;
            for (int q = 0; q < 3; ++q) { se.f[q] = e3[q]; se.f[3 + q] = h[q]; es.f[q] = eo[q]; }
            zp<6, KIND_EH>("k_zpv_EH", 9.0 * N * sizeof(T), se, es);
            Ef = eo;
            hx(Ef, 3);
        } else {
            Ef = passes3<0u>("k_zpv_E", E[0], E[1], 4, true);
        }
        // right-hand side: hydro part (xdif 0..3, 7) and induction (xdif 4..6)
        dim3 gg(mx / ZTX, (my + 7) / 8, 1);
        int ch = zchunk(gg.x * gg.y, 32);
        gg.z = (mz + ch - 1) / ch;
        if (!g.viscos && !g.diffu) {   // register-blocked fast path (no viscosity, no diffusion)
            HydroIO<T> hio;
            hio.drho = xs[0]; hio.m1 = xs[1]; hio.m2 = xs[2]; hio.m3 = xs[3]; hio.dp = xs[7];
            hio.j1 = curF[0]; hio.j2 = curF[1]; hio.j3 = curF[2]; hio.b1 = xs[4]; hio.b2 = xs[5]; hio.b3 = xs[6];
            hio.out[0] = K[0]; hio.out[1] = K[1]; hio.out[2] = K[2]; hio.out[3] = K[3]; hio.out[4] = K[7];
            dim3 gh((mx + ZHc::TX - 1) / ZHc::TX, (my + ZH_TY - 1) / ZH_TY, 1);
            int chh = zchunk(gh.x * gh.y, 16);
            gh.z = (mz + chh - 1) / chh;
#ifndef DASHA_NO_TMA
            ZhMaps maps;
            if (!hydro_maps(hio, maps)) launch_err = "cuTensorMapEncodeTiled failed for the hydro ring";
            DASHA_LAUNCH("k_rhs_hydro", 16.0 * N * sizeof(T),
                         (k_zhydro_tma<T, ZH_VX, ZH_TY, 1, ZH_MINB><<<gh, 32 * ZH_TY, ZHc::smem_tma(), st>>>(g, hio, chh, maps)));
#else
            DASHA_LAUNCH("k_rhs_hydro", 16.0 * N * sizeof(T),
                         (k_zhydro<T, ZH_VX, ZH_TY, 1, ZH_MINB><<<gh, 32 * ZH_TY, ZHc::smem(), st>>>(g, hio, chh)));
#endif
        } else {
        SrcFields<T, 5> sh;
        sh.f[0] = xs[0]; sh.f[1] = xs[1]; sh.f[2] = xs[2]; sh.f[3] = xs[3]; sh.f[4] = xs[7];
        OpHydro<T> oh;
        oh.out[0] = K[0]; oh.out[1] = K[1]; oh.out[2] = K[2]; oh.out[3] = K[3]; oh.out[4] = K[7];
        oh.j1 = curF[0]; oh.j2 = curF[1]; oh.j3 = curF[2]; oh.b1 = xs[4]; oh.b2 = xs[5]; oh.b3 = xs[6];
        DASHA_LAUNCH("k_rhs_hydro", 16.0 * N * sizeof(T),
                     (k_zst2<T, 5, ZTX, 8, HMINB, OpHydro<T>><<<gg, ZTX * 8, ZS2<T, 5, ZTX, 8>::smem(true), st>>>(g, sh, oh, ch)));
        }
        T* kb[3] = {K[4], K[5], K[6]};
        zcurl<-1>("k_rhs_induction", src3(Ef), f3(kb));
        hx(K, 8);
    }
    // 8 scratch fields that are free once the RHS is written
    void tmp8(T** t) {
        T* s[8] = {cur[0][0], cur[0][1], cur[0][2], cur[1][0], cur[1][1], cur[1][2], Hh[0][0], Hh[0][1]};
        for (int m = 0; m < 8; ++m) t[m] = s[m];
    }

    // xdif of state xs into `out` (dasha_rhs): the RHS and, when smoothing, 2 avrg passes
    void launch_rhs(T* const* xs, bool smooth_xdif, T** out) {
        launch_rhs_raw(xs);
        if (smooth_xdif) {
            T* t[8];
            tmp8(t);
            pass8("k_zpv_X", 16.0, K, [&](int lo) { return st4(t, lo); });
            pass8("k_zpv_X", 16.0, t, [&](int lo) { return st4(out, lo); });
        } else {
            for (int m = 0; m < 8; ++m) out[m] = K[m];
        }
    }

    Status stepon(double time, double dt, int nstep) override {
        (void)time;
        NvtxRange range("stepon");
        // stages 1..4: base = X, stage state in S, accumulator in A; both xdif smoothing
        // passes run in one k_zpv2 launch per field pair that ends in the RK stage update.  When
        // the post-step filter runs, its last launch (fields B, p) also takes the CFL rate of the
        // new state for the next setdt (the tap leaves that launch's registers unchanged; on the
        // RK stage-4 launch it would lower occupancy, so a step without the filter leaves setdt
        // its own sweep).
        const int every = P.filter_every > 0 ? P.filter_every : 1;
        const bool filt = nstep % every == 0;
        // a z-slab takes setdt's rate by its own sweep (the tap would also read the ghost planes)
        const bool tap = !cut();
        rate_ok = false;
        hx(X, 8);
        for (int stage = 1; stage <= 4; ++stage) {
            launch_rhs_raw(stage == 1 ? X : S);
            rk_passes(stage, dt, K, X, S, A, KAHAN ? C : nullptr);
        }
        for (int m = 0; m < 8; ++m) std::swap(X[m], S[m]);
        if (filt) {   // avrgtt on the perturbation (t3dsdsc.f:1135-1165)
            T* t[8];
            tmp8(t);
            hx(X, 8);
            if constexpr (KAHAN) {
                hx(C, 8);
                filter_compensated(t, tap);
            } else {
                pass8("k_zpv_F", 16.0, X, [&](int lo) { return st4(t, lo); });
                hx(t, 8);
                SrcFields<T, 4> a, b;
                for (int q = 0; q < 4; ++q) { a.f[q] = t[q]; b.f[q] = t[4 + q]; }
                zp<4, 0u>("k_zpv_F", 8.0 * N * sizeof(T), a, st4(S, 0));
                if (tap) zp<4, KIND_B4>("k_zpv_F", 8.0 * N * sizeof(T) + tap_bytes(), b, with_cfl(st4(S, 4), S));
                else zp<4, KIND_B4>("k_zpv_F", 8.0 * N * sizeof(T), b, st4(S, 4));
                for (int m = 0; m < 8; ++m) std::swap(X[m], S[m]);
            }
        }
        if (nstep % 10 == 0) {      // diagn blow-up guard (t3dsdsc.f:1174-1182, 1232)
            hx(X + 4, 3);           // the current reads B at z-neighbours
            Status s = launch_diag(true);
            if (s.code) return s;
        }
        DASHA_CK(cudaGetLastError());
        if (launch_err) {
            const char* e = launch_err;
            launch_err = nullptr;
            return Status::err(DASHA_E_CUDA, e);
        }
        rate_ok = filt && tap;
        return Status::ok();
    }

    Status launch_diag(bool guard_only) {
        launch_current(X);
        double* rows = red;
        double* fl = red + 2L * my * mz;
        double* jext = fl + my;
        double* out = red + nred;
        (void)guard_only;
        // the planes this context accounts for and its planes of the central z plane(s): all of
        // them on a whole grid; on a z-slab its own planes (and the walls it holds), and the
        // flux where it owns the (first) central plane, the second one an own or ghost plane
        int klo = 0, khi = mz - 1, ka, kb;
        {
            const int mg = halo ? halo->geo.mzg : mz, z0 = halo ? halo->geo.zfirst - 2 : 0;
            if (halo && halo->geo.lower()) klo = 2;
            if (halo && halo->geo.upper()) khi = mz - 3;
            const int ga = mg % 2 ? (mg - 1) / 2 : mg / 2 - 1, gb = mg % 2 ? ga : mg / 2;
            const bool own = ga - z0 >= klo && ga - z0 <= khi;
            ka = own ? ga - z0 : -1;
            kb = own ? gb - z0 : -1;
        }
        dim3 g2(1, my, mz);
        DASHA_LAUNCH("k_diag_rows", 8.0 * N * sizeof(T),
                     k_diag_rows<T><<<g2, 128, 0, st>>>(g, f8(X), wx, wy, wz, P.gamma, rows, klo, khi));
        k_diag_flux<T><<<my, 128, 0, st>>>(g, f8(X), wx, fl, ka, kb);
        k_diag_jext<T><<<mz, 128, 0, st>>>(g, f3(curF), my / 2, jext, klo, khi);
        k_diag_final<<<1, 256, 0, st>>>(rows, (long)my * mz, fl, my, jext, mz, out, flag);
        DASHA_CK(cudaGetLastError());
        return Status::ok();
    }

    Status diagnostics(double* outh) override {
        hx(X + 4, 3);   // a z-slab: the current and a central plane may read B's ghost planes
        Status s = launch_diag(false);
        if (s.code) return s;
        DASHA_CK(cudaMemcpyAsync(hpin, red + nred, sizeof(double) * DASHA_NDIAG, cudaMemcpyDeviceToHost, st));
        DASHA_CK(cudaStreamSynchronize(st));
        if (launch_err) {
            const char* e = launch_err;
            launch_err = nullptr;
            return Status::err(DASHA_E_CUDA, e);
        }
        for (int q = 0; q < DASHA_NDIAG; ++q) outh[q] = hpin[q];
        int none = 0;
        if (halo && halo->per_process() && !halo->reduce_diag(outh, &none))
            return Status::err(DASHA_E_CUDA, "slab diagnostics reduction: " + halo->err);
        return Status::ok();
    }

    Status setdt(double* dt, int* blowup) override {
        NvtxRange range("setdt");
        if (rate_ok) {   // the rate of this state was taken by the last stepon's final launch
            DASHA_CK(cudaMemcpyAsync(hpin + 12, rate_bits, sizeof(double), cudaMemcpyDeviceToHost, st));
            DASHA_CK(cudaMemcpyAsync(hpin + 13, flag, sizeof(int), cudaMemcpyDeviceToHost, st));
            DASHA_CK(cudaStreamSynchronize(st));
            const double v = hpin[12];
            int fl = 0;
            std::memcpy(&fl, hpin + 13, sizeof(int));
            *dt = (v != v) ? v : std::fmin(100.0, 1.0 / v);   // as k_reduce_rate
            *blowup = fl;
            return slab_reduce(dt, blowup);
        }
        dim3 g2(1, my, mz);
        const long nt = (long)mx + my + mz;
        DASHA_LAUNCH("k_cfl", 8.0 * N * sizeof(T),
                     k_cfl_rate<T><<<g2, 128, 0, st>>>(g, f8(X), cfltab, cfltab + nt, cfltab + 2 * nt, P.gamma,
                                                       (P.dt_whistler && P.hall) ? P.di * 3.141592653589793 : 0.0, red));
        k_reduce_rate<<<1, 256, 0, st>>>(red, (long)my * mz, red + nred + 12);
        DASHA_CK(cudaGetLastError());
        DASHA_CK(cudaMemcpyAsync(hpin + 12, red + nred + 12, sizeof(double), cudaMemcpyDeviceToHost, st));
        int fl = 0;
        DASHA_CK(cudaMemcpyAsync(hpin + 13, flag, sizeof(int), cudaMemcpyDeviceToHost, st));
        DASHA_CK(cudaStreamSynchronize(st));
        std::memcpy(&fl, hpin + 13, sizeof(int));
        *dt = hpin[12];
        *blowup = fl;
        return slab_reduce(dt, blowup);
    }
    // a slab of a one-process-per-GPU run: the smallest dt and any blow-up of all slabs (the
    // group entry points of the slabs of one process reduce on the host)
    Status slab_reduce(double* dt, int* blowup) {
        if (halo && halo->per_process() && !halo->reduce(dt, blowup))
            return Status::err(DASHA_E_CUDA, "slab dt reduction: " + halo->err);
        return Status::ok();
    }

    Status current(double* curh, long ld1, long ld2) override {
        hx(X + 4, 3);
        launch_current(X);
        DASHA_CK(cudaGetLastError());
        if (launch_err) {
            const char* e = launch_err;
            launch_err = nullptr;
            return Status::err(DASHA_E_CUDA, e);
        }
        return transfer_out(curh, ld1, ld2, curF, 3, false);
    }

    // The fields of the reference's 2-D output (recrd2, t3dsdsc.f:4965-5113) on the plane
    // j = my/2: one kernel gathers them from the state and the freshly smoothed current, and
    // only mx*mz*11 values cross to the host.
    Status midplane(double* outh) override {
        if (!mpd) DASHA_CK(cudaMalloc(&mpd, sizeof(double) * 11 * (size_t)mx * mz));
        launch_current(X);
        F8<T> cz;
        for (int m = 0; m < 8; ++m) cz.f[m] = KAHAN ? C[m] : nullptr;
        k_midplane<T><<<dim3((mx + 127) / 128, mz), 128, 0, st>>>(g, my / 2, f8(X), cz, f3(curF), mpd);
        DASHA_CK(cudaGetLastError());
        DASHA_CK(cudaMemcpyAsync(outh, mpd, sizeof(double) * 11 * (size_t)mx * mz, cudaMemcpyDeviceToHost, st));
        DASHA_CK(cudaStreamSynchronize(st));
        return Status::ok();
    }

    Status current_out(const ChunkOut& take) override {
        launch_current(X);
        DASHA_CK(cudaGetLastError());
        return stream_out(curF, 3, false, nullptr, take);
    }

    Status rhs(double t, double* xdif, long ld1, long ld2) override {
        T* out[8];
        for (int m = 0; m < 8; ++m) out[m] = S[m];
        launch_rhs(X, t != 0.0, out);
        DASHA_CK(cudaGetLastError());
        return transfer_out(xdif, ld1, ld2, out, 8, false);
    }

    // ======================= discrete adjoint (FP64 contexts) =======================
    // scratch of one adjoint call (cudaMalloc'd per call, freed at the end)
    // scratch of one adjoint call: one cudaMalloc carved into fields (freed at the end)
    struct AdjBufs {
        char* base = nullptr;
        size_t cap = 0, used = 0;
        bool reserve(size_t bytes) {
            if (cudaMalloc((void**)&base, bytes) != cudaSuccess) { cudaGetLastError(); base = nullptr; return false; }
            cap = bytes;
            return true;
        }
        double* take(size_t n) {
            size_t b = (n * sizeof(double) + 255) & ~(size_t)255;
            if (!base || used + b > cap) return nullptr;
            double* p = (double*)(base + used);
            used += b;
            return p;
        }
        ~AdjBufs() { if (base) cudaFree(base); }
    };
    static size_t adj_field_bytes(long n) { return ((size_t)n * sizeof(double) + 255) & ~(size_t)255; }
    struct V8 { T* f[8]; };

    void k8(T** d, T* const* s2) { for (int m = 0; m < 8; ++m) d[m] = s2[m]; }
    void copy8(T* const* dst, T* const* src) {
        DASHA_LAUNCH("a_copy8", 16.0 * N * sizeof(T),
                     for (int m = 0; m < 8; ++m) cudaMemcpyAsync(dst[m], src[m], sizeof(T) * N, cudaMemcpyDeviceToDevice, st));
    }
    void zero8(T* const* f, int nf = 8) { for (int m = 0; m < nf; ++m) cudaMemsetAsync(f[m], 0, sizeof(T) * N, st); }
    void axpby8(T* const* y, double b, T* const* x, double a) {
        if constexpr (std::is_same<T, double>::value) {
            long nb = (N + 255) / 256;
            F8<double> Y, Xv;
            for (int m = 0; m < 8; ++m) { Y.f[m] = y[m]; Xv.f[m] = x[m]; }
            DASHA_LAUNCH("a_axpby", 24.0 * N * 8, k_axpby8<<<nb, 256, 0, st>>>(N, Y, b, Xv, a));
        }
    }

    // the forward step in explicit buffers: stage states S1..S3, result Xo (filtered if
    // filt); same kernels and arithmetic as stepon
    void fwd_step(T* const* Xb, double dt, bool filt, T* const* S1, T* const* S2, T* const* S3, T* const* Xo, T* const* Acc) {
        T* const* outs[4] = {S1, S2, S3, Xo};
        T* const* ins[4] = {Xb, S1, S2, S3};
        for (int stage = 1; stage <= 4; ++stage) {
            launch_rhs_raw(ins[stage - 1]);
            rk_passes(stage, dt, K, Xb, outs[stage - 1], Acc, nullptr);
        }
        if (filt) {
            T* t[8];
            tmp8(t);
            pass8("k_zpv_F", 16.0, Xo, [&](int lo) { return st4(t, lo); });
            pass8("k_zpv_F", 16.0, t, [&](int lo) { return st4(Xo, lo); });
        }
    }

    // transposed smoothing passes: n passes of nf (3 or 8) fields, kinds per field, in place
    // on `a` using `b` as the other buffer; returns the buffer holding the result
    T** adj_passes(T** a, T** b, int nf, int n, unsigned kinds3, bool fold_after) {
        if constexpr (std::is_same<T, double>::value) {
            dim3 gf((mx + blk.x - 1) / blk.x, my, 1);
            for (int p = 0; p < n; ++p) {   // each transposed pass folds its input rows itself
                if (nf == 3) {
                    FS<double, 3> in, out;
                    for (int m = 0; m < 3; ++m) { in.f[m] = a[m]; out.f[m] = b[m]; }
                    DASHA_LAUNCH("a_pass3", 6.0 * N * 8, k_adj_pass<3><<<grd, blk, 0, st>>>(g, adj_cr, in, out, kinds3));
                } else {
                    FS<double, 4> in, out;
                    for (int m = 0; m < 4; ++m) { in.f[m] = a[m]; out.f[m] = b[m]; }
                    DASHA_LAUNCH("a_pass4", 8.0 * N * 8, k_adj_pass<4><<<grd, blk, 0, st>>>(g, adj_cr, in, out, 0u));
                    for (int m = 0; m < 4; ++m) { in.f[m] = a[4 + m]; out.f[m] = b[4 + m]; }
                    DASHA_LAUNCH("a_pass4", 8.0 * N * 8, k_adj_pass<4><<<grd, blk, 0, st>>>(g, adj_cr, in, out, KIND_B4));
                }
                std::swap(a, b);
            }
            if (fold_after) {
                F8<double> fa{};
                for (int m = 0; m < nf; ++m) fa.f[m] = a[m];
                k_adj_fold_rows<<<dim3((mx + blk.x - 1) / blk.x, my, 1), blk, 0, st>>>(g, fa, nf);
            }
        }
        return a;
    }

    // sigma = G'(S)^T kappa, G = avrg(right(.)); eta partials summed into *eta_acc (device)
    struct AdjScratch {
        T *a8[8], *b8[8], *sb[8], *wq[8];
        T *e0[3], *e1[3], *et[3], *h0[3], *h1[3], *jb[3], *jt[3], *ub[3];
        double* etap;
        long netap;
        double* eta_acc;
    };
    void adj_rhs(T* const* Sx, T* const* kappa, T* const* sigma, AdjScratch& w) {
        if constexpr (std::is_same<T, double>::value) {
            launch_current(Sx);                       // curF = J of the stage state
            for (int m = 0; m < 8; ++m) cudaMemcpyAsync(w.a8[m], kappa[m], sizeof(T) * N, cudaMemcpyDeviceToDevice, st);
            T** rb = adj_passes(w.a8, w.b8, 8, 2, 0u, true);       // adjoint of the raw RHS (rows folded)
            // induction: o_B = -curl(E_total)  ->  Et_bar = -curl^T(o_B)
            F3<double> ob3, et3;
            for (int m = 0; m < 3; ++m) { ob3.f[m] = rb[4 + m]; et3.f[m] = w.et[m]; }
            DASHA_LAUNCH("a_curlT", 6.0 * N * 8, k_adj_curlT<<<grd, blk, 0, st>>>(g, ob3, et3, -1.0, 0));
            // E chain: 4 transposed avrgE passes -> adjoint of E0 (all nodes)
            for (int m = 0; m < 3; ++m) cudaMemcpyAsync(w.e0[m], w.et[m], sizeof(T) * N, cudaMemcpyDeviceToDevice, st);
            T** eb = adj_passes(w.e0, w.e1, 3, 4, 0u, false);
            T** hb = nullptr;
            if (P.hall) {   // Hall chain: 5 transposed avrgh passes, then the rows of the Hall field (k_zeh) folded
                for (int m = 0; m < 3; ++m) cudaMemcpyAsync(w.h0[m], w.et[m], sizeof(T) * N, cudaMemcpyDeviceToDevice, st);
                hb = adj_passes(w.h0, w.h1, 3, 5, KIND_H, true);
            }
            zero8(w.sb);
            AdjPtw ap;
            for (int m = 0; m < 8; ++m) { ap.s.f[m] = Sx[m]; ap.sb.f[m] = w.sb[m]; ap.wq.f[m] = w.wq[m]; }
            for (int m = 0; m < 3; ++m) {
                ap.j.f[m] = curF[m]; ap.eb.f[m] = eb[m]; ap.hb.f[m] = hb ? hb[m] : w.et[m];
                ap.jb.f[m] = w.jb[m]; ap.ub.f[m] = w.ub[m];
            }
            ap.ob[0] = rb[0]; ap.ob[1] = rb[1]; ap.ob[2] = rb[2]; ap.ob[3] = rb[3]; ap.ob[4] = rb[7];
            ap.etapart = w.etap;
            ap.hall = P.hall;
            DASHA_LAUNCH("a_pointwise", 30.0 * N * 8, k_adj_pointwise<<<grd, blk, 0, st>>>(g, ap));
            DASHA_LAUNCH("a_reduce", 0.0, k_reduce_add<<<1, 256, 0, st>>>(w.etap, w.netap, w.eta_acc));
            AdjGat ag;
            for (int m = 0; m < 8; ++m) { ag.s.f[m] = Sx[m]; ag.sb.f[m] = w.sb[m]; ag.wq.f[m] = w.wq[m]; }
            for (int m = 0; m < 3; ++m) ag.ub.f[m] = w.ub[m];
            ag.ob[0] = rb[0]; ag.ob[1] = rb[1]; ag.ob[2] = rb[2]; ag.ob[3] = rb[3]; ag.ob[4] = rb[7];
            DASHA_LAUNCH("a_gather", 25.0 * N * 8, k_adj_gather<<<grd, blk, 0, st>>>(g, ag));
            // current chain: 4 transposed avrgc passes, the curl's rows folded, curl^T into B
            T** jt = adj_passes(w.jb, w.jt, 3, 4, 0u, true);
            F3<double> jw, bo;
            for (int m = 0; m < 3; ++m) { jw.f[m] = jt[m]; bo.f[m] = w.sb[4 + m]; }
            DASHA_LAUNCH("a_curlT", 9.0 * N * 8, k_adj_curlT<<<grd, blk, 0, st>>>(g, jw, bo, 1.0, 1));
            for (int m = 0; m < 8; ++m) cudaMemcpyAsync(sigma[m], w.sb[m], sizeof(T) * N, cudaMemcpyDeviceToDevice, st);
        }
    }

    long w_netap_max() const { return (long)grd.x * grd.y * grd.z; }
    double* adj_cr = nullptr;   // radial coefficient field of the current adjoint call
    bool adj_scratch(AdjBufs& B, AdjScratch& w) {
        if constexpr (std::is_same<T, double>::value) {
            if (!(adj_cr = B.take(N))) return false;
            k_adj_cr<<<grd, blk, 0, st>>>(g, adj_cr);
        }
        auto t8 = [&](T** a) { for (int m = 0; m < 8; ++m) if (!(a[m] = (T*)B.take(N))) return false; return true; };
        auto t3 = [&](T** a) { for (int m = 0; m < 3; ++m) if (!(a[m] = (T*)B.take(N))) return false; return true; };
        if (!t8(w.a8) || !t8(w.b8) || !t8(w.sb) || !t8(w.wq)) return false;
        if (!t3(w.e0) || !t3(w.e1) || !t3(w.et) || !t3(w.h0) || !t3(w.h1) || !t3(w.jb) || !t3(w.jt) || !t3(w.ub)) return false;
        w.netap = (long)grd.x * grd.y * grd.z;
        if (!(w.etap = B.take(w.netap)) || !(w.eta_acc = B.take(4))) return false;
        cudaMemsetAsync(w.eta_acc, 0, 4 * sizeof(double), st);
        return true;
    }

    Status adjoint_rhs(const double* wh, double* outh, long ld1, long ld2) override {
        if constexpr (!std::is_same<T, double>::value) {
            (void)wh; (void)outh; (void)ld1; (void)ld2;
            return Status::err(DASHA_E_UNSUPPORTED, "the adjoint runs on FP64 contexts only");
        } else {
            if (g.viscos || g.diffu) return Status::err(DASHA_E_UNSUPPORTED, "adjoint with viscous/diffusive terms");
            AdjBufs B;
            AdjScratch w;
            T *kap[8], *sig[8];
            if (!B.reserve(adj_field_bytes(N) * (60 + 16) + adj_field_bytes(w_netap_max()) + 4096))
                return Status::err(DASHA_E_NOMEM, "adjoint scratch");
            if (!adj_scratch(B, w)) return Status::err(DASHA_E_NOMEM, "adjoint scratch");
            for (int m = 0; m < 8; ++m) {
                if (!(kap[m] = (T*)B.take(N)) || !(sig[m] = (T*)B.take(N))) return Status::err(DASHA_E_NOMEM, "adjoint scratch");
            }
            Status s2 = transfer_in(wh, ld1, ld2, kap, 8, false);
            if (s2.code) return s2;
            adj_rhs(X, kap, sig, w);
            DASHA_CK(cudaGetLastError());
            return transfer_out(outh, ld1, ld2, sig, 8, false);
        }
    }

    // Reverse sweep of one step j: the stage states of step j are in s1..s3, Xn is state j;
    // lambda (in lam) goes from dPhi/dX_{j+1} to dPhi/dX_j.
    // mu = F^T lambda (the post-step filter when step j filtered), then the RK4 stages in reverse:
    // kappa4 = dt/6 mu, sigma3 = G'(S3)^T kappa4, kappa3 = dt/3 mu + dt sigma3, ...,
    // lambda = mu + sigma0 + sigma1 + sigma2 + sigma3.
    struct AdjVec { T *lam[8], *mu[8], *kap[8], *sig[8], *tot[8], *ta[8], *tb[8]; };
    void adj_step(T* const* Xn, T* const* s1, T* const* s2, T* const* s3, double dt, bool filtered, AdjVec& v,
                  AdjScratch& w) {
        if (filtered) {
            copy8(v.ta, v.lam);
            T** r = adj_passes(v.ta, v.tb, 8, 2, 0u, false);
            copy8(v.mu, r);
        } else {
            copy8(v.mu, v.lam);
        }
        copy8(v.tot, v.mu);                                    // lambda_X = mu + sum sigma
        copy8(v.kap, v.mu);
        axpby8(v.kap, dt / 6.0, v.mu, 0.0);                    // kappa4 = dt/6 mu
        adj_rhs(s3, v.kap, v.sig, w);                          // sigma3
        axpby8(v.tot, 1.0, v.sig, 1.0);
        axpby8(v.kap, 0.0, v.mu, dt / 3.0);                    // kappa3 = dt/3 mu + dt sigma3
        axpby8(v.kap, 1.0, v.sig, dt);
        adj_rhs(s2, v.kap, v.sig, w);                          // sigma2
        axpby8(v.tot, 1.0, v.sig, 1.0);
        axpby8(v.kap, 0.0, v.mu, dt / 3.0);                    // kappa2 = dt/3 mu + dt/2 sigma2
        axpby8(v.kap, 1.0, v.sig, dt / 2.0);
        adj_rhs(s1, v.kap, v.sig, w);                          // sigma1
        axpby8(v.tot, 1.0, v.sig, 1.0);
        axpby8(v.kap, 0.0, v.mu, dt / 6.0);                    // kappa1 = dt/6 mu + dt/2 sigma1
        axpby8(v.kap, 1.0, v.sig, dt / 2.0);
        adj_rhs(Xn, v.kap, v.sig, w);                          // sigma0
        axpby8(v.tot, 1.0, v.sig, 1.0);
        copy8(v.lam, v.tot);
    }
    // the seed lambda = dPhi/dX_N of the reconnected flux of the final state X_N
    void adj_seed(T* const* XN, T* const* lam) {
        zero8(lam);
        dim3 g2((mx + blk.x - 1) / blk.x, my, 1);
        k_adj_flux_seed<<<g2, blk, 0, st>>>(g, XN[6], wx, lam[6]);
    }

    Status adjoint_flux_grad(int nsteps, const double* dts, int snaps, double* deta, double* dpsi) override {
        if constexpr (!std::is_same<T, double>::value) {
            (void)nsteps; (void)dts; (void)snaps; (void)deta; (void)dpsi;
            return Status::err(DASHA_E_UNSUPPORTED, "the adjoint runs on FP64 contexts only");
        } else {
            if (g.viscos || g.diffu) return Status::err(DASHA_E_UNSUPPORTED, "adjoint with viscous/diffusive terms");
            const int every = P.filter_every > 0 ? P.filter_every : 1;
            AdjBufs B;
            AdjScratch w;
            // fields: scratch 60, 13 work vectors of 8, then either every step and stage state
            // of the run (keep-all) or the binomial plan's state slots
            size_t freeb = 0, totb = 0;
            cudaMemGetInfo(&freeb, &totb);
            const size_t fb = adj_field_bytes(N);
            const size_t extra = adj_field_bytes(w_netap_max()) + adj_field_bytes((long)mx * mz) + 8192;
            const double budget = 0.85 * (double)freeb;
            const size_t fixed_fields = 60 + 13 * 8;
            // snaps == 0: keep every step and stage state of the forward sweep when they fit (one
            // forward sweep, nothing recomputed), else the binomial plan with as many state slots
            // as fit; snaps > 0: the binomial plan with `snaps` free state slots
            const size_t all_fields = fixed_fields + (size_t)(nsteps + 1) * 8 + 24 * (size_t)nsteps;
            const bool keep_all = snaps == 0 && (double)(all_fields * fb + extra) < budget;
            if (snaps == 0 && !keep_all) {
                const double room = (budget - (double)(extra + (fixed_fields + 16) * fb)) / (8.0 * (double)fb);
                if (room < 1.0) return Status::err(DASHA_E_NOMEM, "adjoint checkpoints do not fit in device memory");
                snaps = (int)std::min<double>(room, std::max(1, nsteps - 1));
            }
            if (!keep_all) snaps = std::max(1, std::min(snaps, std::max(1, nsteps - 1)));
            const size_t want = keep_all ? all_fields * fb + extra : (fixed_fields + 16 + 8 * (size_t)snaps) * fb + extra;
            if (!B.reserve(want)) return Status::err(DASHA_E_NOMEM, "adjoint checkpoints do not fit in device memory");
            if (!adj_scratch(B, w)) return Status::err(DASHA_E_NOMEM, "adjoint scratch");
            auto take8 = [&](T** a) { for (int m = 0; m < 8; ++m) if (!(a[m] = (T*)B.take(N))) return false; return true; };
            T *X0[8], *S1[8], *S2[8], *S3[8], *Xo[8], *Ac[8];
            AdjVec v;
            bool ok = take8(X0) && take8(S1) && take8(S2) && take8(S3) && take8(Xo) && take8(Ac) && take8(v.lam) &&
                      take8(v.mu) && take8(v.kap) && take8(v.sig) && take8(v.tot) && take8(v.ta) && take8(v.tb);
            if (!ok) return Status::err(DASHA_E_NOMEM, "adjoint checkpoints do not fit in device memory");
            copy8(X0, X);
            if (keep_all) {
                // every step state and its stage states from one forward sweep
                std::vector<std::vector<T*>> sst(nsteps + 1, std::vector<T*>(8)), stg(3L * nsteps, std::vector<T*>(8));
                for (auto& q : sst) ok = ok && take8(q.data());
                for (auto& q : stg) ok = ok && take8(q.data());
                if (!ok) return Status::err(DASHA_E_NOMEM, "adjoint stage states");
                copy8(sst[0].data(), X0);
                for (int n = 0; n < nsteps; ++n)
                    fwd_step(sst[n].data(), dts[n], n % every == 0, stg[3 * n].data(), stg[3 * n + 1].data(),
                             stg[3 * n + 2].data(), sst[n + 1].data(), Ac);
                adj_seed(sst[nsteps].data(), v.lam);
                for (int n = nsteps - 1; n >= 0; --n)
                    adj_step(sst[n].data(), stg[3 * n].data(), stg[3 * n + 1].data(), stg[3 * n + 2].data(), dts[n],
                             n % every == 0, v, w);
            } else {
                // binomial checkpointing (checkpoint_schedule.h): slot 0 holds state 0, slots
                // 1..snaps are free; reversing step j re-runs step j from state j for its stage
                // states (the last step's run also gives the final state, and with it the seed)
                std::vector<std::vector<T*>> slot(snaps + 1, std::vector<T*>(8));
                T *cur[8], *nxt[8];
                ok = take8(cur) && take8(nxt);
                for (int q = 1; q <= snaps; ++q) ok = ok && take8(slot[q].data());
                if (!ok) return Status::err(DASHA_E_NOMEM, "adjoint checkpoints do not fit in device memory");
                for (int m = 0; m < 8; ++m) slot[0][m] = X0[m];
                copy8(cur, X0);
                for (const CkptAction& a : binomial_schedule(nsteps, snaps)) {
                    switch (a.kind) {
                        case CkptAction::Restore: copy8(cur, slot[a.a].data()); break;
                        case CkptAction::Store: copy8(slot[a.a].data(), cur); break;
                        case CkptAction::Release: break;
                        case CkptAction::Advance:
                            for (int j = a.a; j < a.b; ++j) {
                                fwd_step(cur, dts[j], j % every == 0, S1, S2, S3, nxt, Ac);
                                std::swap_ranges(cur, cur + 8, nxt);
                            }
                            break;
                        case CkptAction::Reverse: {
                            const int j = a.a;
                            fwd_step(cur, dts[j], j % every == 0, S1, S2, S3, Xo, Ac);
                            if (j == nsteps - 1) adj_seed(Xo, v.lam);
                            adj_step(cur, S1, S2, S3, dts[j], j % every == 0, v, w);
                            break;
                        }
                    }
                }
            }
            // gradients: eta, and psi through dBx = -Dz psi, dBz = Dx psi
            double* dpsi_d = B.take((size_t)mx * mz);
            if (!dpsi_d) return Status::err(DASHA_E_NOMEM, "adjoint scratch");
            k_adj_psi<<<dim3((mx + blk.x - 1) / blk.x, mz, 1), blk, 0, st>>>(g, v.lam[4], v.lam[6], dpsi_d);
            DASHA_CK(cudaGetLastError());
            std::vector<double> hp((size_t)mx * mz);
            DASHA_CK(cudaMemcpyAsync(hp.data(), dpsi_d, sizeof(double) * mx * mz, cudaMemcpyDeviceToHost, st));
            double he = 0.0;
            DASHA_CK(cudaMemcpyAsync(&he, w.eta_acc, sizeof(double), cudaMemcpyDeviceToHost, st));
            copy8(X, X0);                                              // the context state is unchanged
            rate_ok = false;
            DASHA_CK(cudaStreamSynchronize(st));
            *deta = he;
            std::memcpy(dpsi, hp.data(), sizeof(double) * mx * mz);
            return Status::ok();
        }
    }
};

// one chunk of whole z planes k0.. (compact mx x my x nk doubles) into / out of field T
template <class T>
__global__ void k_import_chunk(int mx, int my, int k0, const double* src, const double* eqprof, T* dst) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= mx) return;
    const int j = blockIdx.y, k = k0 + blockIdx.z;
    double v = src[(long)i + (long)mx * (j + (long)my * blockIdx.z)];
    if (eqprof) v -= eqprof[k];
    dst[(long)i + (long)mx * (j + (long)my * k)] = T(v);
}
template <class T>
__global__ void k_export_chunk(int mx, int my, int k0, const T* src, const T* comp, const double* eqprof, double* dst) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= mx) return;
    const int j = blockIdx.y, k = k0 + blockIdx.z;
    const long n = (long)i + (long)mx * (j + (long)my * k);
    double v = (double)src[n];
    if (comp) v -= (double)comp[n];   // compensated FP32 state: the value is x - comp
    if (eqprof) v += eqprof[k];
    dst[(long)i + (long)mx * (j + (long)my * blockIdx.z)] = v;
}

// out[q][k][i], q = rho, (rho v)/rho, B, p (FP64 totals, formed as k_export_chunk forms them),
// then the current density; one thread per (i, k) on the plane j
template <class T>
__global__ void k_midplane(Geo<T> g, int j, F8<T> x, F8<T> comp, F3<T> cur, double* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y;
    if (i >= g.mx) return;
    const long n = (long)i + (long)g.mx * (j + (long)g.my * k);
    const long np = (long)g.mx * g.mz, o = (long)i + (long)g.mx * k;
    const double* prof[8] = {g.rho0, nullptr, nullptr, nullptr, g.bx0, g.by0, g.bz0, g.p0};
    double v[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) {
        v[m] = (double)x.f[m][n];
        if (comp.f[m]) v[m] -= (double)comp.f[m][n];
        if (prof[m]) v[m] += prof[m][k];
    }
    out[o] = v[0];
#pragma unroll
    for (int m = 1; m < 4; ++m) out[m * np + o] = v[m] / v[0];
#pragma unroll
    for (int m = 4; m < 8; ++m) out[m * np + o] = v[m];
#pragma unroll
    for (int m = 0; m < 3; ++m) out[(8 + m) * np + o] = (double)cur.f[m][n];
}

template <class T>
inline const double* eq_profile(const Geo<T>& g, int m) {
    switch (m) {
        case 0: return g.rho0;
        case 4: return g.bx0;
        case 5: return g.by0;
        case 6: return g.bz0;
        case 7: return g.p0;
        default: return nullptr;
    }
}

}  // namespace dasha
