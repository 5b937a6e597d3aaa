/*
 * The reference program on nprx x nprz ranks, each rank a thread -- TEST INFRASTRUCTURE ONLY.
 *
 * Built by oracle/refmodel.py as
 *     gcc -DREF_TLS=__thread -DREF_GENERATED='"<translated reference>.c"' ref_ranks.c mpi_threads.c
 * so that this file sees the translated program's COMMON blocks (one copy per thread).  Each
 * thread does what one MPI rank of the reference does: the main program's process set-up
 * (t3dsdsc.f:33-81), `input` on the global grid given here in place of gridpntnew2 (it slices
 * its own nodes and exchanges their halo with message1), then the given equilibrium and state on
 * its own nodes and halo, foreta / formu, and the main loop's setdt + stepon (t3dsdsc.f:136-175).
 * Rank 0 times the K timed steps between barriers.  Arrays from the caller are C-order numpy:
 * the state (8, mz, my, mx), profiles (mz), coordinates; out_state (8, mz, my, mx) receives
 * every rank's own nodes after the run.
 */
#include REF_GENERATED
#include <pthread.h>
#include <time.h>

void mpt_set_rank(int r);
void mpt_init(int n);
void mpt_fini(void);
void mpt_barrier(void);

typedef struct {
    int nprx, nprz, mx, my, mz, warm, steps, hall;
    const double *xc, *yc, *zc, *state, *rho0, *bx0, *by0, *bz0, *p0;
    double eta, cht, cfl, time0;
    double* out_state;
    double* seconds;
    double* dts;
} job;

static job J;

static double now(void) {
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

#define A3(a, jx, jy, jz, ld1, ld2) (a)[((jx) - 1) + (long)(ld1) * (((jy) - 1) + (long)(ld2) * ((jz) - 1))]

static void* rank_main(void* arg) {
    const int r = (int)(long)arg;
    mpt_set_rank(r);
    const int nprx = J.nprx, nprz = J.nprz, mx = J.mx, my = J.my, mz = J.mz;
    const int mxpr = mx / nprx + 4, mzpr = mz / nprz + 4;
    /* t3dsdsc.f:33-81 */
    cb_indexmpi.nrank = r;
    cb_indexmpi.nsize = nprx * nprz;
    int left = r - 1, right = r + 1, low = r - nprx, up = r + nprx;
    if (left % nprx == nprx - 1 || left < 0) left = -2;
    if (right % nprx == 0) right = -2;
    if (low < 0) low = -2;
    if (up > nprx * nprz - 1) up = -2;
    cb_indexmpi.myleft = left; cb_indexmpi.myright = right; cb_indexmpi.mylow = low; cb_indexmpi.myupper = up;
    const int mepx = r % nprx, mepz = r / nprx;
    cb_indexmpi.mepx = mepx; cb_indexmpi.mepz = mepz;
    cb_indexmpi.xfirst = 3; cb_indexmpi.xlast = mxpr - 2; cb_indexmpi.zfirst = 3; cb_indexmpi.zlast = mzpr - 2;
    if (mepx == nprx - 1) cb_indexmpi.xlast = mxpr - 2 + mx % nprx;
    if (mepz == nprz - 1) cb_indexmpi.zlast = mzpr - 2 + mz % nprz;
    cb_indexmpi.x_first = 3; cb_indexmpi.x_last = mxpr - 2; cb_indexmpi.z_first = 3; cb_indexmpi.z_last = mzpr - 2;
    if (mepx == 0) cb_indexmpi.x_first = 5;
    if (mepx == nprx - 1) cb_indexmpi.x_last = mxpr - 4 + mx % nprx;
    if (mepz == 0) cb_indexmpi.z_first = 5;
    if (mepz == nprz - 1) cb_indexmpi.z_last = mzpr - 4 + mz % nprz;
    cb_run.dtstatus = 1; cb_run.nst = 1; cb_run.nstnew = 1;
    /* the global grid in place of gridpntnew2: nodes and forward spacings */
    for (int i = 0; i < mx; ++i) {
        cb_var16.xxt[i] = J.xc[i];
        cb_var16.dxt[i] = i + 1 < mx ? J.xc[i + 1] - J.xc[i] : J.xc[i] - J.xc[i - 1];
    }
    for (int j = 0; j < my; ++j) {
        cb_var15.yy[j] = J.yc[j];
        cb_var15.dy[j] = j + 1 < my ? J.yc[j + 1] - J.yc[j] : J.yc[j] - J.yc[j - 1];
    }
    for (int k = 0; k < mz; ++k) {
        cb_var16.zzt[k] = J.zc[k];
        cb_var16.dzt[k] = k + 1 < mz ? J.zc[k + 1] - J.zc[k] : J.zc[k] - J.zc[k - 1];
    }
    f_input();
    cb_cst.eta0 = J.eta; cb_para3.rcr = -1.0; cb_logic.hall = J.hall; cb_cst.cfl = J.cfl;
    cb_cst.time = J.time0; cb_run.nstep = 1;
    ref_cht_value = J.cht;
    /* equilibrium, state and radius on this rank's nodes and halo (global node gx = mepx (mxpr-4)
     * + jx - 2, 1-based; halo beyond the domain left zero) */
    const long N = (long)mx * my * mz;
    for (int jz = 1; jz <= mzpr; ++jz) {
        const int gz = mepz * (mzpr - 4) + jz - 2;
        if (gz < 1 || gz > mz) continue;
        for (int jy = 1; jy <= my; ++jy)
            for (int jx = 1; jx <= mxpr; ++jx) {
                const int gx = mepx * (mxpr - 4) + jx - 2;
                if (gx < 1 || gx > mx) continue;
                const long g = (long)(gx - 1) + (long)mx * ((jy - 1) + (long)my * (gz - 1));
                for (int m = 0; m < 8; ++m)
                    cb_var21.x[((jx - 1) + (long)mxpr * ((jy - 1) + (long)my * ((jz - 1) + (long)mzpr * m)))] = J.state[m * N + g];
                A3(cb_var11.rhoi, jx, jy, jz, mxpr, my) = J.rho0[gz - 1];
                A3(cb_var11.bxi, jx, jy, jz, mxpr, my) = J.bx0[gz - 1];
                A3(cb_wrk.byi, jx, jy, jz, mxpr, my) = J.by0[gz - 1];
                A3(cb_var11.bzi, jx, jy, jz, mxpr, my) = J.bz0[gz - 1];
                A3(cb_var11.pri, jx, jy, jz, mxpr, my) = J.p0[gz - 1];
                const double rr = sqrt(J.xc[gx - 1] * J.xc[gx - 1] + J.yc[jy - 1] * J.yc[jy - 1] + J.zc[gz - 1] * J.zc[gz - 1]);
                A3(cb_wrk.rr0, jx, jy, jz, mxpr, my) = rr;
                A3(cb_wrk.rr1, jx, jy, jz, mxpr, my) = rr;
            }
    }
    double t = J.time0;
    f_foreta(&t);
    f_formu(&t);
    double t0 = 0.0;
    for (int n = 0; n < J.warm + J.steps; ++n) {
        if (n == J.warm) { mpt_barrier(); t0 = now(); }
        f_setdt();
        if (r == 0 && J.dts) J.dts[n] = cb_cst.dt;
        f_stepon();
        cb_run.nstep += 1;
        cb_cst.time += cb_cst.dt;
    }
    mpt_barrier();
    if (r == 0 && J.seconds) *J.seconds = now() - t0;
    if (J.out_state) {   /* this rank's own nodes */
        for (int jz = cb_indexmpi.zfirst; jz <= cb_indexmpi.zlast; ++jz)
            for (int jy = 1; jy <= my; ++jy)
                for (int jx = cb_indexmpi.xfirst; jx <= cb_indexmpi.xlast; ++jx) {
                    const int gx = mepx * (mxpr - 4) + jx - 2, gz = mepz * (mzpr - 4) + jz - 2;
                    const long g = (long)(gx - 1) + (long)mx * ((jy - 1) + (long)my * (gz - 1));
                    for (int m = 0; m < 8; ++m)
                        J.out_state[m * N + g] = cb_var21.x[((jx - 1) + (long)mxpr * ((jy - 1) + (long)my * ((jz - 1) + (long)mzpr * m)))];
                }
    }
    return NULL;
}

/* Runs warm + steps steps of the reference on nprx x nprz thread ranks; the decomposition must
 * be the one this file was built for.  Returns 0. */
int ref_ranks_run(int nprx, int nprz, int mx, int my, int mz, const double* xc, const double* yc, const double* zc,
                  const double* state, const double* rho0, const double* bx0, const double* by0, const double* bz0,
                  const double* p0, double eta, double cht, int hall, double cfl, int warm, int steps,
                  double* out_state, double* seconds, double* dts) {
    J.nprx = nprx; J.nprz = nprz; J.mx = mx; J.my = my; J.mz = mz; J.warm = warm; J.steps = steps; J.hall = hall;
    J.xc = xc; J.yc = yc; J.zc = zc; J.state = state; J.rho0 = rho0; J.bx0 = bx0; J.by0 = by0; J.bz0 = bz0; J.p0 = p0;
    J.eta = eta; J.cht = cht; J.cfl = cfl; J.time0 = 0.0;
    J.out_state = out_state; J.seconds = seconds; J.dts = dts;
    const int n = nprx * nprz;
    mpt_init(n);
    pthread_t th[1024];
    pthread_attr_t at;
    pthread_attr_init(&at);
    pthread_attr_setstacksize(&at, (size_t)64 << 20);
    for (int r = 0; r < n; ++r) pthread_create(&th[r], &at, rank_main, (void*)(long)r);
    for (int r = 0; r < n; ++r) pthread_join(th[r], NULL);
    pthread_attr_destroy(&at);
    mpt_fini();
    return 0;
}
