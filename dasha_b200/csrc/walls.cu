// walls.cu -- the engine of the reference's own bounded configuration (walls_core.cuh): a
// context created with periodic = {0, 0, 0}.  FP64, one thread per node for every loop of the
// reference's routines, on the reference's padded local layout.  Built with -fmad=false: the
// reference's expressions are rounded as written (no contraction to FMA), so the results follow
// the reference's own arithmetic to the rounding of the transcendental functions.
#include "dasha_capi.h"
#include "engine.cuh"
#include "walls_core.cuh"

#include <cstring>
#include <vector>

namespace dasha {

namespace {

using walls::Box;

template <class F>
__global__ void k_walls(Box b, F f) {
    const int jx = b.x0 + (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (jx > b.x1) return;
    f(jx, b.y0 + (int)blockIdx.y, b.z0 + (int)blockIdx.z);
}

struct GpuExec {
    cudaStream_t st;
    template <class F>
    void run(Box b, F f) {
        if (b.x1 < b.x0 || b.y1 < b.y0 || b.z1 < b.z0) return;
        const dim3 grid((unsigned)((b.x1 - b.x0 + 1 + 127) / 128), (unsigned)(b.y1 - b.y0 + 1), (unsigned)(b.z1 - b.z0 + 1));
        k_walls<<<grid, 128, 0, st>>>(b, f);
    }
    // the minimum of positive doubles through their bit patterns (ordered as unsigned integers)
    __host__ __device__ static void atomic_min_bits(unsigned long long* p, double v) {
#ifdef __CUDA_ARCH__
        atomicMin(p, (unsigned long long)__double_as_longlong(v));
#else
        (void)p; (void)v;
#endif
    }
};

class WallEngine : public EngineBase {
public:
    GpuExec ex{};
    walls::Dims d{};
    walls::Par par{};
    walls::Arr a{};
    walls::Tables t{};
    void* pool = nullptr;
    double* tab = nullptr;
    cudaStream_t st = nullptr;
    long n = 0;
    std::vector<double> hx;          // host staging of one padded 8-field array
    bool eq_set = false;

    ~WallEngine() override {
        if (pool) cudaFree(pool);
        if (tab) cudaFree(tab);
    }
    walls::Core<GpuExec> core() { return walls::Core<GpuExec>{ex, d, t, par, a}; }

    Status init(int mx, int my, int mz, const dasha_params_c& p, cudaStream_t st_, const double* xc, const double* yc,
                const double* zc) {
        st = st_;
        ex.st = st_;
        d = walls::make_dims(mx, my, mz);
        n = d.n;
        par.gamma = p.gamma; par.eta = p.eta; par.mu = p.viscos ? p.mu : 0.; par.drho = p.diffu ? p.drho : 0.;
        par.dp = p.diffu ? p.dp : 0.; par.cfl = p.cfl; par.rcr = p.rcr; par.chall = p.di;
        par.hall = p.hall; par.viscos = p.viscos; par.diffu = p.diffu; par.uyzlimiter = p.uyzlimiter;
        DASHA_CK(cudaMalloc(&pool, sizeof(double) * n * walls::NFIELDS + 256));
        DASHA_CK(cudaMemsetAsync(pool, 0, sizeof(double) * n * walls::NFIELDS + 256, st));
        DASHA_CK(cudaStreamSynchronize(st));          // the stream does not order with the copies below
        double* q = static_cast<double*>(pool);
        walls::carve(a, [&](int k) { double* r = q; q += (size_t)k * n; return r; });
        a.dtbits = reinterpret_cast<unsigned long long*>(q);
        // the 1-D tables, concatenated in one device buffer
        const std::vector<std::vector<double>> tabs = walls::make_tables(d, xc, yc, zc);
        std::vector<double> ht;
        std::vector<size_t> off;
        for (const auto& v : tabs) { off.push_back(ht.size()); ht.insert(ht.end(), v.begin(), v.end()); }
        DASHA_CK(cudaMalloc(&tab, sizeof(double) * ht.size()));
        DASHA_CK(cudaMemcpy(tab, ht.data(), sizeof(double) * ht.size(), cudaMemcpyHostToDevice));
        const double* tp[walls::NTAB];
        for (int k = 0; k < walls::NTAB; ++k) tp[k] = tab + off[k];
        walls::bind_tables(t, tp);
        {
            const std::vector<double> r = walls::make_radius(d, tabs);
            DASHA_CK(cudaMemcpy(a.rr0, r.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
            DASHA_CK(cudaMemcpy(a.rr1, r.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
        }
        hx.assign(8 * (size_t)n, 0.);
        DASHA_CK(cudaStreamSynchronize(st));
        return Status::ok();
    }

    // physical nodes of a host array in the reference's layout (leading dimensions ld1, ld2,
    // (i+2) + ld1 (j + ld2 ((k+2) + (mz+4) m))) to / from the padded device array
    void host_to_pad(const double* src, long ld1, long ld2, int nf, double* dst) const {
        for (int m = 0; m < nf; ++m)
            for (int k = 0; k < d.mz; ++k)
                for (int j = 0; j < d.my; ++j)
                    std::memcpy(dst + m * n + d.at(3, j + 1, k + 3), src + 2 + ld1 * (j + ld2 * ((k + 2) + (long)(d.mz + 4) * m)),
                                sizeof(double) * d.mx);
    }
    void pad_to_host(const double* src, long ld1, long ld2, int nf, double* dst) const {
        for (int m = 0; m < nf; ++m)
            for (int k = 0; k < d.mz; ++k)
                for (int j = 0; j < d.my; ++j)
                    std::memcpy(dst + 2 + ld1 * (j + ld2 * ((k + 2) + (long)(d.mz + 4) * m)), src + m * n + d.at(3, j + 1, k + 3),
                                sizeof(double) * d.mx);
    }
    Status upload(double* dev, int nf) {
        DASHA_CK(cudaMemcpyAsync(dev, hx.data(), sizeof(double) * nf * n, cudaMemcpyHostToDevice, st));
        DASHA_CK(cudaStreamSynchronize(st));
        return Status::ok();
    }
    Status download(const double* dev, int nf) {
        DASHA_CK(cudaMemcpyAsync(hx.data(), dev, sizeof(double) * nf * n, cudaMemcpyDeviceToHost, st));
        DASHA_CK(cudaStreamSynchronize(st));
        return Status::ok();
    }

    // the equilibrium, then xresd as initia computes it (T:805-834): the state set to the
    // equilibrium, right(0, 1e-9, 1) with eta = 0 (foreta runs after it), xresd = the momentum rates
    Status equilibrium_from_hx() {
        Status s = upload(a.xm, 5);                   // rho0 bx0 by0 bz0 p0 staged in xm
        if (s.code) return s;
        double* eq[5] = {a.rhoi, a.bxi, a.byi, a.bzi, a.pri};
        for (int q = 0; q < 5; ++q) DASHA_CK(cudaMemcpyAsync(eq[q], a.xm + q * n, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
        const int from[8] = {0, -1, -1, -1, 1, 2, 3, 4};
        for (int m = 0; m < 8; ++m) {
            if (from[m] < 0) DASHA_CK(cudaMemsetAsync(a.x + m * n, 0, sizeof(double) * n, st));
            else DASHA_CK(cudaMemcpyAsync(a.x + m * n, eq[from[m]], sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
        }
        DASHA_CK(cudaMemcpyAsync(a.xfold, a.x, sizeof(double) * 8 * n, cudaMemcpyDeviceToDevice, st));
        DASHA_CK(cudaMemsetAsync(a.xresd, 0, sizeof(double) * 3 * n, st));
        const double eta = par.eta;
        par.eta = 0.;
        core().right(0., 1.e-9, 1);
        par.eta = eta;
        DASHA_CK(cudaMemcpyAsync(a.xresd, a.xdif + n, sizeof(double) * 3 * n, cudaMemcpyDeviceToDevice, st));
        DASHA_CK(cudaGetLastError());
        DASHA_CK(cudaStreamSynchronize(st));
        eq_set = true;
        return Status::ok();
    }
    Status set_equilibrium(const double* rho0, const double* b0, const double* p0, const double*) override {
        // z-profiles broadcast over x and y
        std::fill(hx.begin(), hx.end(), 0.);
        const double* prof[5] = {rho0, b0, b0 + d.mz, b0 + 2 * d.mz, p0};
        for (int q = 0; q < 5; ++q)
            for (int k = 0; k < d.mz; ++k)
                for (int j = 1; j <= d.my; ++j)
                    for (int i = 3; i <= d.mx + 2; ++i) hx[q * n + d.at(i, j, k + 3)] = prof[q][k];
        return equilibrium_from_hx();
    }
    Status set_equilibrium_3d(const double* eq, long ld1, long ld2) override {
        std::fill(hx.begin(), hx.end(), 0.);
        host_to_pad(eq, ld1, ld2, 5, hx.data());
        return equilibrium_from_hx();
    }
    Status set_j0(const double*) override { return Status::err(DASHA_E_UNSUPPORTED, "J0 is a periodic-context option"); }
    Status set_state(const double* x, long ld1, long ld2) override {
        std::fill(hx.begin(), hx.end(), 0.);
        host_to_pad(x, ld1, ld2, 8, hx.data());
        return upload(a.x, 8);
    }
    Status get_state(double* x, long ld1, long ld2) override {
        Status s = download(a.x, 8);
        if (s.code) return s;
        pad_to_host(hx.data(), ld1, ld2, 8, x);
        return Status::ok();
    }
    Status setdt(double* dt, int* blowup) override {
        const double hundred = 100.;
        unsigned long long bits;
        std::memcpy(&bits, &hundred, sizeof(bits));
        DASHA_CK(cudaMemcpyAsync(a.dtbits, &bits, sizeof(bits), cudaMemcpyHostToDevice, st));
        core().setdt_launch();
        DASHA_CK(cudaGetLastError());
        DASHA_CK(cudaMemcpyAsync(&bits, a.dtbits, sizeof(bits), cudaMemcpyDeviceToHost, st));
        DASHA_CK(cudaStreamSynchronize(st));
        std::memcpy(dt, &bits, sizeof(double));
        *blowup = 0;
        return Status::ok();
    }
    Status stepon(double time, double dt, int) override {
        NvtxRange range("stepon (bounded)");
        core().stepon(time, dt);
        DASHA_CK(cudaGetLastError());
        return Status::ok();
    }
    Status current(double* cur, long ld1, long ld2) override {
        core().current();
        DASHA_CK(cudaGetLastError());
        Status s = download(a.cur, 3);
        if (s.code) return s;
        pad_to_host(hx.data(), ld1, ld2, 3, cur);
        return Status::ok();
    }
    // right(t, 1e-9, 1) with xfold = x, as initia calls it; the state is restored afterwards
    // (the inflow driver writes the x-min rows of x)
    Status rhs(double tt, double* xdif, long ld1, long ld2) override {
        DASHA_CK(cudaMemcpyAsync(a.xfold, a.x, sizeof(double) * 8 * n, cudaMemcpyDeviceToDevice, st));
        core().right(tt, 1.e-9, 1);
        DASHA_CK(cudaMemcpyAsync(a.x, a.xfold, sizeof(double) * 8 * n, cudaMemcpyDeviceToDevice, st));
        DASHA_CK(cudaGetLastError());
        Status s = download(a.xdif, 8);
        if (s.code) return s;
        pad_to_host(hx.data(), ld1, ld2, 8, xdif);
        return Status::ok();
    }
    static Status no(const char* what) {
        return Status::err(DASHA_E_UNSUPPORTED, std::string(what) + " is not available on a bounded (periodic 0,0,0) context");
    }
    Status state_in(const ChunkIn&) override { return no("streamed state transfer"); }
    Status state_out(const ChunkOut&) override { return no("streamed state transfer"); }
    Status current_out(const ChunkOut&) override { return no("streamed current transfer"); }
    int raw_fields() const override { return 8; }
    size_t raw_elem() const override { return sizeof(double); }
    Status raw_out(const std::function<bool(const void*, size_t)>&) override { return no("the exact-resume record"); }
    Status raw_in(const std::function<bool(void*, size_t)>&) override { return no("the exact-resume record"); }
    Status midplane(double*) override { return no("dasha_midplane"); }
    Status diagnostics(double*) override { return no("dasha_diagnostics"); }
    Status adjoint_flux_grad(int, const double*, int, double*, double*) override { return no("the adjoint"); }
    Status adjoint_rhs(const double*, double*, long, long) override { return no("the adjoint"); }
};

}  // namespace

EngineBase* make_engine_walls(int mx, int my, int mz, const dasha_params_c& p, cudaStream_t st, const double* x,
                              const double* y, const double* z, Status& s) {
    WallEngine* e = new WallEngine();
    s = e->init(mx, my, mz, p, st, x, y, z);
    if (s.code) { delete e; return nullptr; }
    return e;
}

}  // namespace dasha
