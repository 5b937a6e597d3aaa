// Test build of the bounded-configuration core (dasha_b200/csrc/walls_core.cuh) for the host:
// the same loops and arithmetic as the device engine, run by a host executor, for bit-for-bit
// comparison with the translated reference program (tests/test_walls_host.py).
//
// Two checks of the properties the device executor relies on:
//  - order: every loop runs forward, backward or in a shuffled node order; the device runs the
//    nodes of a loop concurrently, so the result must not depend on the order;
//  - guard: every field and every 1-D table sits between PROT_NONE guard pages, its data flush
//    with the start of its pages or with their end, so any access outside an array faults here,
//    on the host.
#include "walls_core.cuh"

#include <sys/mman.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

using namespace dasha::walls;

namespace {

int g_order = 0;       // 0 forward, 1 backward, 2 shuffled
bool g_end = false;    // data flush with the end of its pages

struct HostExec {
    template <class F>
    void run(Box b, F f) {
        const int nx = b.x1 - b.x0 + 1, ny = b.y1 - b.y0 + 1, nz = b.z1 - b.z0 + 1;
        if (nx <= 0 || ny <= 0 || nz <= 0) return;
        if (g_order == 0) {
            for (int jz = b.z0; jz <= b.z1; ++jz)
                for (int jy = b.y0; jy <= b.y1; ++jy)
                    for (int jx = b.x0; jx <= b.x1; ++jx) f(jx, jy, jz);
        } else if (g_order == 1) {
            for (int jz = b.z1; jz >= b.z0; --jz)
                for (int jy = b.y1; jy >= b.y0; --jy)
                    for (int jx = b.x1; jx >= b.x0; --jx) f(jx, jy, jz);
        } else {
            std::vector<int> idx((size_t)nx * ny * nz);
            for (size_t i = 0; i < idx.size(); ++i) idx[i] = (int)i;
            static unsigned s = 12345u;
            for (size_t i = idx.size(); i > 1; --i) {
                s = s * 1103515245u + 12345u;
                std::swap(idx[i - 1], idx[(s >> 8) % i]);
            }
            for (int q : idx) f(b.x0 + q % nx, b.y0 + (q / nx) % ny, b.z0 + q / (nx * ny));
        }
    }
    static void atomic_min_bits(unsigned long long* p, double v) {
        unsigned long long b;
        std::memcpy(&b, &v, sizeof(b));
        if (b < *p) *p = b;
    }
};

const long PG = 4096 / 8;    // doubles per page
long rup(long v) { return (v + PG - 1) / PG * PG; }

// nf arrays of S doubles at a common stride, each between PROT_NONE guard pages of G doubles
double* guarded(long S, int nf, long G, long* stride) {
    const long R = rup(S);
    *stride = R + G;
    const long total = G + nf * (R + G);
    void* m = mmap(nullptr, total * 8, PROT_READ | PROT_WRITE, MAP_PRIVATE | MAP_ANONYMOUS, -1, 0);
    if (m == MAP_FAILED) { perror("mmap"); abort(); }
    double* b = static_cast<double*>(m);
    mprotect(b, G * 8, PROT_NONE);
    for (int q = 0; q < nf; ++q) mprotect(b + G + q * (R + G) + R, G * 8, PROT_NONE);
    return b + G + (g_end ? R - S : 0);
}

struct Ctx {
    HostExec ex;
    Dims d;
    Par par;
    Arr a;
    Tables t;
    long S;                    // doubles of one padded field
    unsigned long long bits;
    Core<HostExec> core() { return Core<HostExec>{ex, d, t, par, a}; }
};

void copy_fields(double* dst, long dst_st, const double* src, long src_st, int nf, long S) {
    for (int m = 0; m < nf; ++m) std::memcpy(dst + m * dst_st, src + m * src_st, sizeof(double) * S);
}

}  // namespace

extern "C" {

// Arrays on the caller's side are the padded layout, S = (mx+4)*my*(mz+4) doubles per field.
void* wh_create(int mx, int my, int mz, const double* xc, const double* yc, const double* zc, const double* par,
                int hall, int uyzlimiter, int order, int guard_end) {
    g_order = order;
    g_end = guard_end != 0;
    Ctx* h = new Ctx();
    h->d = make_dims(mx, my, mz);
    h->S = h->d.n;
    const long G = rup(3 * h->d.sz + 64);    // guards wider than any stencil reach (2 planes)
    long stride = 0;
    guarded(h->S, 1, G, &stride);            // the stride every field array shares
    h->d.n = stride;                         // field m of an array at m * stride
    h->par = Par{par[0], par[1], par[2], par[3], par[4], par[5], par[6], par[7], hall, 1, 1, uyzlimiter};
    carve(h->a, [&](int k) { long st; return guarded(h->S, k, G, &st); });
    h->a.dtbits = &h->bits;
    const std::vector<std::vector<double>> tabs = make_tables(make_dims(mx, my, mz), xc, yc, zc);
    const double* tp[NTAB];
    for (int k = 0; k < NTAB; ++k) {
        long st;
        double* g = guarded((long)tabs[k].size(), 1, PG, &st);
        std::memcpy(g, tabs[k].data(), sizeof(double) * tabs[k].size());
        tp[k] = g;
    }
    bind_tables(h->t, tp);
    const std::vector<double> r = make_radius(make_dims(mx, my, mz), tabs);
    std::memcpy(h->a.rr0, r.data(), sizeof(double) * h->S);
    std::memcpy(h->a.rr1, r.data(), sizeof(double) * h->S);
    return h;
}

// the equilibrium (rhoi bxi byi bzi pri), then initia's state and xresd (T:805-834)
void wh_set_eq(void* hp, const double* eq) {
    Ctx* h = static_cast<Ctx*>(hp);
    const long n = h->d.n, S = h->S;
    Arr& a = h->a;
    double* e[5] = {a.rhoi, a.bxi, a.byi, a.bzi, a.pri};
    for (int q = 0; q < 5; ++q) std::memcpy(e[q], eq + q * S, sizeof(double) * S);
    const int from[8] = {0, -1, -1, -1, 1, 2, 3, 4};
    for (int m = 0; m < 8; ++m) {
        if (from[m] < 0) std::memset(a.x + m * n, 0, sizeof(double) * S);
        else std::memcpy(a.x + m * n, e[from[m]], sizeof(double) * S);
    }
    copy_fields(a.xfold, n, a.x, n, 8, S);
    for (int m = 0; m < 3; ++m) std::memset(a.xresd + m * n, 0, sizeof(double) * S);
    const double eta = h->par.eta;
    h->par.eta = 0.;
    h->core().right(0., 1.e-9, 1);
    h->par.eta = eta;
    copy_fields(a.xresd, n, a.xdif + n, n, 3, S);
}

void wh_set_x(void* hp, const double* x) {
    Ctx* h = static_cast<Ctx*>(hp);
    copy_fields(h->a.x, h->d.n, x, h->S, 8, h->S);
}

// which: 0 x (8 fields), 1 cur (3), 2 xresd (3)
void wh_get(void* hp, int which, double* out) {
    Ctx* h = static_cast<Ctx*>(hp);
    const double* src = which == 0 ? h->a.x : (which == 1 ? h->a.cur : h->a.xresd);
    copy_fields(out, h->S, src, h->d.n, which == 0 ? 8 : 3, h->S);
}

double wh_setdt(void* hp) {
    Ctx* h = static_cast<Ctx*>(hp);
    const double hundred = 100.;
    std::memcpy(&h->bits, &hundred, sizeof(double));
    h->core().setdt_launch();
    double dt;
    std::memcpy(&dt, &h->bits, sizeof(double));
    return dt;
}

void wh_stepon(void* hp, double time, double dt) { static_cast<Ctx*>(hp)->core().stepon(time, dt); }
void wh_current(void* hp) { static_cast<Ctx*>(hp)->core().current(); }

}  // extern "C"
