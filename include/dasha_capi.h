/*
 * dasha_capi.h -- C-ABI of libdasha.so, the B200 (sm_100a) RK4 Hall-MHD step.
 *
 * The reference program (t3dsdsc.f) advances its state with two argument-less Fortran
 * subroutines called from its main loop:
 *     call setdt     (t3dsdsc.f:139,  body t3dsdsc.f:4694-4810)
 *     call stepon    (t3dsdsc.f:171,  body t3dsdsc.f:1063-1185)
 * and reads the current density through COMMON /var11/ cur after `call current`
 * (t3dsdsc.f:2452-2500).  All data moves through COMMON blocks (mhd01.for:55-66,
 * mhd02.for:1-6).  This header replaces those bodies: the state lives on the GPU inside an
 * opaque context, and the Fortran loop calls the functions below through an ISO_C_BINDING
 * interface.
 *
 * Conventions
 *  - Every function returns 0 (DASHA_OK) or a DASHA_E_* code; no exception or exit() crosses
 *    the ABI.  The text of the last error of a context is given by dasha_last_error().
 *  - Host pointers are borrowed for the duration of a call only; copies finish before return.
 *  - One host thread per context.  Kernels run in order on the context's own CUDA stream.
 *  - Host state arrays use the reference's layout x(mxpr,my,mzpr,8) at a 1x1 process grid:
 *    Fortran order, x fastest, a 2-node halo in x and z (mxpr = mx+4, mzpr = mz+4), none in
 *    y.  ld1 (>= mx+4) and ld2 (>= my) are the first two leading dimensions; the third is
 *    always mz+4.  Physical node (i,j,k), 0-based, is element
 *        (i+2) + ld1*( j + ld2*( (k+2) + (mz+4)*m ) ),   m = 0..7 = rho, rho*v(3), B(3), p.
 *    Halo entries are ignored on input and left untouched on output.
 *  - x and y are periodic (true wrap); z is bounded by walls whose two outer node rows
 *    follow the reference's fixed rows (t3dsdsc.f:1821-1857).
 */
#ifndef DASHA_CAPI_H
#define DASHA_CAPI_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct dasha_ctx dasha_ctx;

enum {
    DASHA_OK = 0,
    DASHA_E_INVALID = 1,      /* bad argument (null pointer, size, leading dimension) */
    DASHA_E_UNSUPPORTED = 2,  /* an option the library does not implement: periodicity other than
                                 {1,1,0} or {0,0,0}, on a periodic context mx not a multiple of 4
                                 (of 32 with viscosity or diffusion on) or rcr > 0, FP32 on a
                                 bounded one, total_e != 1, the adjoint on an FP32 context, or a
                                 call a bounded context does not offer */
    DASHA_E_CUDA = 3,         /* a CUDA runtime error; the context should be destroyed */
    DASHA_E_NOMEM = 4,        /* the grid does not fit in device memory */
    DASHA_E_DT_COLLAPSE = 5,  /* dt < 0.1*dt0 or not finite: the guard of t3dsdsc.f:142-154 */
    DASHA_E_BLOWUP = 6,       /* max Jy on the mid-y plane >= 1e7: the guard of t3dsdsc.f:1232 */
    DASHA_E_STATE = 7,        /* call out of order (no equilibrium or state set yet) */
    DASHA_E_NOSCRATCH = 8     /* a size beyond a fixed scratch limit */
};

/* Grid: node coordinates (FP64, host, borrowed).  Replaces gridpntnew2 (t3dsdsc.f:4380-4690)
 * and the local slices of input (t3dsdsc.f:296-313).  periodic:
 *  {1,1,0}  the build's Harris configurations: x and y periodic (a true wrap), z walls; FP64 or
 *           the FP32 perturbation form; the fast z-marching kernels;
 *  {0,0,0}  the reference's own bounded configuration (periodx = periody = periodz = .false.,
 *           mhd03.for), the dipole magnetosphere of initia: walls on all six sides with the rows
 *           of bndry / bndrytt / bndryc / bndryh / bndryE, the time-dependent inflow driver on
 *           the x-min rows (T:1710-1773), the inner-sphere mask r <= rcr, the radial Hall
 *           coefficient 0.5 di (tanh((r-1.1)/8) - tanh((r-2)/10)) (T:1398; di is chall), setdt
 *           over the cells with r >= 1 and a 3-D equilibrium (dasha_set_equilibrium_3d).  FP64
 *           only; the post-step filter every step as in the reference; the streamed transfers,
 *           exact-resume record, mid-plane, diagnostics and adjoint are not offered
 *           (DASHA_E_UNSUPPORTED). */
typedef struct {
    int mx, my, mz;
    const double *x, *y, *z;
    int periodic[3];
} dasha_grid_c;

/* Run-time constants and flags, mhd03.for:1-83 and COMMON /cst/ (mhd01.for:55).
 *  gamma, cfl                      mhd03.for:60,71
 *  eta (etan = eta0), mu (fmu0), drho (frho0), dp (fpr0)   foreta/formu t3dsdsc.f:6489-6532
 *  di: Hall coefficient cht: uniform on periodic contexts; on bounded contexts the reference's
 *    radial profile of it (t3dsdsc.f:1398)
 *  rcr: inner-sphere mask radius (mhd03.for:26); on periodic contexts only rcr <= 0 (no mask)
 *  hall, viscos, diffu, total_e: mhd03.for:18-23 (total_e must be 1)
 *  j0_mode: 0 = LITERAL (J = curl(B-B0), the reference's equations), 1 = FULL (J0 added)
 *  filter_every: cadence of the post-step filter avrgtt (reference: every step = 1)
 *  precision: 0 = FP64 state and arithmetic; 1 = FP32 perturbation + Kahan-compensated RK4
 *  dt_whistler: 0 = the reference's CFL (fast speed only, t3dsdsc.f:4719-4733); 1 = also add
 *    the grid-scale whistler speed di*pi*|B|/(rho*h) to each direction's signal speed (the
 *    explicit Hall term is unstable at fine grids without it; no counterpart in the reference)
 *  uyzlimiter: the reference's uy/uz limiter (mhd03.for:22, .false. there): after bndry and
 *    bndrytt, the z momentum of the two wall rows at each z end and the y momentum of the two
 *    rows at each y end may only point into the domain (t3dsdsc.f:1928-1975, 2231-2278).
 *    Bounded contexts only; 1 on a periodic context returns DASHA_E_UNSUPPORTED */
typedef struct {
    double gamma, eta, di, mu, drho, dp, cfl, rcr;
    int hall, viscos, diffu, total_e, j0_mode;
    int filter_every;
    int precision;
    int dt_whistler;
    int uyzlimiter;
} dasha_params_c;

#define DASHA_NDIAG 9

/* Create a context on the current CUDA device: copies the grid, builds the stencil
 * coefficients (input, t3dsdsc.f:336-606) and allocates all device buffers. */
int dasha_create(const dasha_grid_c* grid, const dasha_params_c* params, dasha_ctx** out);

/* Equilibrium as FP64 1-D z-profiles, length mz each: rho0, b0 = [bx0|by0|bz0] (3*mz), p0.
 * Replaces the 3-D COMMON arrays rhoi, bxi, byi, bzi, pri (t3dsdsc.f:805-813) and computes
 * the residual xresd of the pure equilibrium (t3dsdsc.f:816-834). */
int dasha_set_equilibrium(dasha_ctx* ctx, const double* rho0, const double* b0, const double* p0);

/* A 3-D equilibrium: rho0, bx0, by0, bz0, p0 as 5 fields in the state layout (leading
 * dimensions ld1 >= mx+4, ld2 >= my as in dasha_set_state), replacing the COMMON arrays rhoi,
 * bxi, byi, bzi, pri that initia sets (t3dsdsc.f:805-813).  Bounded contexts only (periodic =
 * {0,0,0}, below); it also computes xresd as initia does (T:828-834): the momentum rates of
 * right(0, 1e-9, 1) with the state set to the equilibrium and eta = 0.  The state is then the
 * one initia leaves, ready to step: the equilibrium at rest, with the rho, vx and p of the two
 * x-min node rows as that right call's inflow driver wrote them; dasha_set_state replaces it.
 * dasha_set_equilibrium on a bounded context broadcasts its z-profiles over x and y and does
 * the same. */
int dasha_set_equilibrium_3d(dasha_ctx* ctx, const double* eq_f, long ld1, long ld2);

/* J0 = curl B0 as FP64 z-profiles [j0x|j0y|j0z] (3*mz), used when j0_mode = FULL.  Without
 * this call FULL mode takes J0 from the z-derivative of b0 with the 4th-order stencil. */
int dasha_set_equilibrium_current(dasha_ctx* ctx, const double* j0);

/* Upload / download the total state x(mxpr,my,mzpr,8) (COMMON /var21/ x, mhd02.for:4). */
int dasha_set_state(dasha_ctx* ctx, const double* x_f, long ld1, long ld2);
int dasha_get_state(dasha_ctx* ctx, double* x_f, long ld1, long ld2);

/* The restart file of recrd / readin (t3dsdsc.f:4814-4861; the format of dasha_restart_write
 * below) written from, or read into, the context's state without a full host copy: the state
 * streams through the context's pinned chunk buffers, file I/O overlapped with the DMA.
 * dasha_checkpoint writes what dasha_restart_write writes for the dasha_get_state array with
 * the x halo holding the periodic copies and the z halo zeros; max_subrecord as there.
 * dasha_restore checks the file's records against the grid before it replaces the state
 * (a mismatch returns DASHA_E_INVALID with the state unchanged); it needs the equilibrium set
 * and acts as dasha_set_state of the file's interior nodes.  An I/O error during the read
 * leaves the context without a state (DASHA_E_STATE until the next set_state or restore).
 * Exact resume (no counterpart in the reference): the file holds FP64 totals, from which the
 * context's stored state (the perturbation from the equilibrium; in FP32 also its Kahan
 * compensation) can be recovered only to one rounding, so dasha_checkpoint also writes
 * <path>.state, that stored state as it is (a 48-byte header "DASHAST1", int32 precision, mx,
 * my, mz, field count, ncase, nstep, nst, double time; then the fields, node i + mx (j + my k)),
 * and dasha_restore, when <path>.state exists, checks that it belongs to the file and the
 * context (else DASHA_E_INVALID with the state unchanged) and takes the state from it: a run
 * restored that way continues bit for bit.  Without <path>.state the file alone is read. */
int dasha_checkpoint(dasha_ctx* ctx, const char* path, int ncase, int nstep, double time, int nst,
                     long max_subrecord);
int dasha_restore(dasha_ctx* ctx, const char* path, int* ncase, int* nstep, double* time, int* nst);

/* Chunked download, for callers that write their own files without a host copy of the
 * volume: what = 0 streams the state (the 8 fields of dasha_get_state), what = 1 the smoothed
 * current (the 3 fields of dasha_current).  fn(user, m, k0, k1, rows) is called once per chunk,
 * fields in order and z planes in order within a field, rows holding field m on planes
 * k0..k1-1 as (k1-k0)*my rows of mx FP64 values (x fastest, no halo), valid during the call
 * only; the next chunk's transfer runs meanwhile.  A non-zero return stops the transfer
 * (DASHA_E_INVALID).  No counterpart in the reference. */
typedef int (*dasha_chunk_fn)(void* user, int m, int k0, int k1, const double* rows);
int dasha_stream_out(dasha_ctx* ctx, int what, dasha_chunk_fn fn, void* user);

/* The m3d file of recrd3 (the format of dasha_m3d_write below) written from the context through
 * dasha_stream_out: no host copy of the state or the current, only of rho (mx*my*mz values) for
 * v = (rho v)/rho; the coordinates are the grid's.  The text equals dasha_m3d_write of the
 * dasha_get_state and dasha_current arrays. */
int dasha_m3d_write_ctx(dasha_ctx* ctx, const char* path, double time);

/* CFL time step of the current state (setdt, t3dsdsc.f:4694-4763): synchronises, returns dt.
 * Also reports a latched blow-up (DASHA_E_BLOWUP) and dt collapse (DASHA_E_DT_COLLAPSE,
 * dt < 0.1*dt0 with dt0 the first dt of the context, t3dsdsc.f:142). */
int dasha_setdt(dasha_ctx* ctx, double time, double* dt_out);

/* One RK4 step (stepon, t3dsdsc.f:1063-1185), enqueued asynchronously.  nstep is the step
 * counter before the step: the post-step filter runs when nstep % filter_every == 0 and the
 * blow-up guard (diagn) when nstep % 10 == 0. */
int dasha_stepon(dasha_ctx* ctx, double time, double dt, int nstep);

/* Smoothed current density cur(mxpr,my,mzpr,3) of the current state (current,
 * t3dsdsc.f:2452-2500), same layout rules as the state. */
int dasha_current(dasha_ctx* ctx, double* cur_f, long ld1, long ld2);

/* The eleven fields of the reference's 2-D output on the mid-y plane j = my/2 (0-based; nyh =
 * my/2+1 in recrd2, t3dsdsc.f:4965-5113), with the smoothed current of the current state:
 * plane[q*mx*mz + i + mx*k] for q = 0 rho, 1-3 v = (rho v)/rho, 4-6 B, 7 p (totals), 8-10 J.
 * Only this plane crosses to the host; dasha_m2d_write formats it. */
int dasha_midplane(dasha_ctx* ctx, double* plane);

/* One right-hand side xdif(mxpr,my,mzpr,8) = dx/dt of the current state at stage time t
 * (right, t3dsdsc.f:1297-1673); the xdif smoothing avrg runs only when t != 0. */
int dasha_rhs(dasha_ctx* ctx, double t, double* xdif_f, long ld1, long ld2);

/* FP64 diagnostics of the current state, out[DASHA_NDIAG]:
 *  [0] mass  sum(rho dV)      [1] energy  sum((rho v^2/2 + p/(gamma-1) + B^2/2) dV)
 *  [2] reconnected flux  (1/my) sum_y sum_x sqrt(Bz(z=0)^2 + 1e-20) dx
 *  [3..8] Jx max, Jx min, Jy max, Jy min, Jz max, Jz min on the mid-y plane (diagn,
 *  t3dsdsc.f:1189-1235). */
int dasha_diagnostics(dasha_ctx* ctx, double* out);

/* Gradient of the final reconnected flux (out[2] of dasha_diagnostics) after nsteps RK4
 * steps with the recorded dt sequence dt_seq[nsteps], starting from the current state, with
 * respect to eta (*dPhi_deta) and to a psi perturbation on the (x,z) nodes (dPhi_dpsi[mx*mz],
 * x fastest), where the perturbation enters the initial B as dBx = -Dz psi, dBz = Dx psi.
 * snaps > 0: binomial checkpointing (the revolve strategy of Griewank and Walther) with
 * `snaps` free state slots besides the initial state: binomial_cost(nsteps, snaps) forward steps
 * to reach the states the schedule stores (the fewest possible with that many slots), plus one
 * re-run of every step for its stage states as it is reversed; snaps == 0: every step and stage
 * state of one forward sweep is kept when they fit in 85 % of the free device memory (nothing is
 * recomputed), else the binomial plan with as many slots as fit there.  FP64 contexts only.
 * The state of the context is left unchanged. */
int dasha_adjoint_flux_grad(dasha_ctx* ctx, int nsteps, const double* dt_seq, int snaps,
                            double* dPhi_deta, double* dPhi_dpsi);

/* Verification hook of the adjoint (no counterpart in the reference): out = G'(x)^T w, the
 * transposed Jacobian of one smoothed right-hand side G = avrg(right(.)) at the current state,
 * applied to w; both in the state layout (8 fields).  FP64 contexts only. */
int dasha_adjoint_rhs(dasha_ctx* ctx, const double* w_f, double* out_f, long ld1, long ld2);

/* Measurement helpers (no counterpart in the reference).
 * dasha_timer(ctx, 0, NULL) records a start event on the context stream;
 * dasha_timer(ctx, 1, &ms) records a stop event, waits for it and returns the elapsed ms.
 * dasha_profile(ctx, 1) brackets every later kernel launch with CUDA events on the context
 * stream (this slows launches down; use it for breakdowns, not for headline numbers);
 * dasha_profile_read(ctx, n, names, ms, launches, bytes) waits, then fills up to n rows:
 * names (32 chars each), total ms, launch count and the algorithmic bytes of one launch per
 * kernel kind, returns the number of rows in *n, and clears the record. */
int dasha_timer(dasha_ctx* ctx, int op, double* ms);
int dasha_profile(dasha_ctx* ctx, int enable);
int dasha_profile_read(dasha_ctx* ctx, int* n, char* names, double* ms, long* launches, double* bytes);

/* Smoothed current density without any device allocation.  No counterpart in the reference:
 * for callers that cannot call cudaMalloc (their device memory is owned by a pool or a
 * budget, or the allocator must not be called at that point).  Computes what dasha_current
 * computes for j0_mode LITERAL, J = S^4(curl(B - B0)) with the wall rows, from caller device
 * arrays: db_dev = B - B0 and cur_dev = J, each 3 fields of mx*my*mz FP64 values, node
 * (i,j,k) at i + mx*(j + my*k), field stride mx*my*mz; the two 3-field ranges must not
 * overlap (an in-place call returns DASHA_E_INVALID).  Work is enqueued on `stream` (a
 * cudaStream_t, NULL for the default stream).  The ping-pong buffer and the stencil tables
 * live in one static device array of DASHA_NOALLOC_SCRATCH_DOUBLES doubles (about 26 MB) that
 * every GPU loading the library holds until exit; grids above DASHA_NOALLOC_MAX_CELLS nodes
 * or DASHA_NOALLOC_MAX_AXIS nodes per axis return DASHA_E_NOSCRATCH.  The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress); make that first call
 * before any stream capture.  Calls share the array: calls that overlap on the GPU race. */
#define DASHA_NOALLOC_MAX_CELLS (1L << 20)
#define DASHA_NOALLOC_MAX_AXIS 4096
#define DASHA_NOALLOC_SCRATCH_DOUBLES (3L * DASHA_NOALLOC_MAX_CELLS + 3L * 7 * DASHA_NOALLOC_MAX_AXIS)
int dasha_current_noalloc(const dasha_grid_c* grid, const double* db_dev, double* cur_dev, void* stream);

/* ---- z-slab decomposition over several GPUs ----
 * The multi-GPU form of the reference's domain decomposition (mhd01.for:5-6: nprx x nprz MPI
 * ranks, each with a 2-node halo refreshed by message4, t3dsdsc.f:6354-6419), cut in z only:
 * the interior rows 2..mz-3 are split into nslabs slabs of consecutive rows, and slab s is a
 * context over its own rows plus two planes on each side (global rows first-2 .. first+count+1:
 * the wall rows at a global wall, ghost copies of the neighbour's edge rows elsewhere).  The
 * ghost planes are refreshed after every launch whose output a later launch reads at
 * z-neighbours, so every slab's own rows take the values of the one-context run, bit for bit.
 * Periodic (1,1,0) contexts only; the whole-grid calls (dasha_checkpoint, dasha_restore,
 * dasha_stream_out, dasha_m3d_write_ctx, dasha_midplane, dasha_rhs, the adjoint,
 * dasha_set_equilibrium_3d) return DASHA_E_UNSUPPORTED on a slab; dasha_diagnostics reduces
 * over the slabs.
 *
 * dasha_slab_partition: own rows of slab `slab` (host only): count = (mz-4)/nslabs, the first
 *   (mz-4)%nslabs slabs one more; DASHA_E_INVALID unless every slab gets at least 3 rows.
 * dasha_create_slab: grid = the GLOBAL grid; the context is created on the current device.  Its
 *   dasha_set_equilibrium / dasha_set_equilibrium_current take the global profiles (mz values
 *   each) and keep the slab's planes; dasha_set_state / dasha_get_state / dasha_current carry
 *   the slab's local array, mz_local = count + 4 planes (global rows first-2 ..), in the usual
 *   halo layout; the ghost planes of the input are not read.
 * dasha_slab_rows: the slab's first own global row, own row count and local plane count. */
int dasha_slab_partition(int mz, int nslabs, int slab, int* first, int* count);
/* The ghost exchange of slab `slab` (host only), in values of one field whose planes hold `plane`
 * values (mx*my): peer[0] / peer[1] the slab below / above (-1 at a wall); it sends `count`
 * values from send_off[q] to peer[q] and receives `count` values at recv_off[q] from peer[q].
 * The NCCL and the in-process exchanges move exactly these ranges. */
int dasha_slab_halo_plan(int mz, int nslabs, int slab, long plane, int* peer, long* send_off, long* recv_off,
                         long* count);
int dasha_create_slab(const dasha_grid_c* grid, const dasha_params_c* params, int nslabs, int slab, dasha_ctx** out);
int dasha_slab_rows(dasha_ctx* ctx, int* first, int* count, int* mz_local);

/* One process, every slab (one per GPU, or several on one GPU): dasha_slab_link joins
 * ctxs[0..n-1] (slab s at ctxs[s]) into a group whose ghost planes are copied between the
 * slabs' memories (cudaMemcpyPeerAsync, ordered against the neighbours' launches by events, and
 * peer access enabled between neighbouring GPUs).  A linked group steps through the
 * dasha_group_* calls, which run every slab in its own host thread: dasha_group_setdt returns
 * the smallest dt of the slabs (the guards of dasha_setdt apply; it synchronises),
 * dasha_group_stepon enqueues one RK4 step of the whole grid, dasha_group_current writes slab
 * s's current to cur_f[s].  The
 * single-context dasha_setdt / dasha_stepon / dasha_current of a linked slab return
 * DASHA_E_STATE; a slab that is joined to nothing also returns DASHA_E_STATE there. */
int dasha_slab_link(dasha_ctx* const* ctxs, int n);
int dasha_group_setdt(dasha_ctx* const* ctxs, int n, double time, double* dt_out);
int dasha_group_stepon(dasha_ctx* const* ctxs, int n, double time, double dt, int nstep);
int dasha_group_current(dasha_ctx* const* ctxs, int n, double* const* cur_f, long ld1, long ld2);
/* dasha_diagnostics of the whole grid from a linked group: mass, energy and flux summed over the
 * slabs' own planes (and the walls the end slabs hold; the flux from the slab that owns the
 * first central plane), the J extrema over all of them.  A slab of a one-process-per-GPU run
 * takes dasha_diagnostics itself (reduced over the ranks by ncclAllReduce). */
int dasha_group_diagnostics(dasha_ctx* const* ctxs, int n, double* out);

/* One process per GPU, each with one slab (the reference's one MPI rank per process): rank 0
 * makes an NCCL id (dasha_nccl_unique_id, 128 bytes), every rank receives it by its own means
 * (MPI_Bcast, torch.distributed) and joins with dasha_slab_nccl (collective: it returns once
 * all nslabs ranks have joined).  Then each rank calls dasha_setdt / dasha_stepon /
 * dasha_current on its slab as on a whole-grid context; the ghost planes travel by ncclSend /
 * ncclRecv on the context's stream and setdt's dt is the minimum over the ranks
 * (ncclAllReduce).  Every rank must make the same calls in the same order.  NCCL is loaded
 * at run time: the libnccl.so.2 already in the process, else the one the loader finds; without
 * it both calls return DASHA_E_UNSUPPORTED.  A process holds one libnccl.so.2 and libraries
 * loaded later bind to it, so a process that also uses another NCCL user (torch) loads that one
 * first. */
int dasha_nccl_unique_id(void* id, int nbytes);
int dasha_slab_nccl(dasha_ctx* ctx, const void* id, int nbytes);

/* Host-side files of the reference's output routines (no context, no GPU).  Each returns
 * DASHA_OK or DASHA_E_INVALID (bad argument, an I/O error, or a file that does not match).
 *
 * Restart file mhdNNNRRR, the reference's file name for step index nst and rank RRR (000 at the
 * 1x1 process grid): recrd writes it and readin reads it (t3dsdsc.f:4814-4861).  Fortran
 * unformatted sequential, native byte order, gfortran's record markers (4-byte lengths around
 * subrecords of at most 2147483639 bytes; a longer record is split into subrecords, the
 * leading length negative while more follow, the trailing one negative after the first).
 * Record 1: ncase, nstep (INTEGER*4), time (REAL*8), nst (INTEGER*4).  Record 2: the whole
 * array x(mx+4, my, mz+4, 8), halo entries included, taken from (read into) an array with
 * leading dimensions ld1 >= mx+4, ld2 >= my as in dasha_get_state.  max_subrecord: 0 for
 * gfortran's limit, or a smaller subrecord length.  The reader accepts any subrecord split and
 * rejects a record whose length is not the expected one. */
int dasha_restart_write(const char* path, int ncase, int nstep, double time, int nst, int mx, int my, int mz,
                        const double* x_f, long ld1, long ld2, long max_subrecord);
int dasha_restart_read(const char* path, int* ncase, int* nstep, double* time, int* nst, int mx, int my, int mz,
                       double* x_f, long ld1, long ld2);

/* The restart files of an nprx x nprz MPI run of the reference, one per rank:
 * <dir>/mhdNNNRRR, RRR = rank (t3dsdsc.f:36-67, 4814-4861), each the rank's x(mxpr, my, mzpr, 8)
 * with mxpr = mx/nprx + 4, mzpr = mz/nprz + 4 (mhd01.for:5-6), rank r at process coordinates
 * (r mod nprx, r / nprx), the last rank of each direction holding the one extra node when
 * mx mod nprx (mz mod nprz) is 1; the reference allows no larger remainder.
 * dasha_restart_read_ranks assembles the global state (interior nodes of every rank) into the
 * dasha_set_state layout, checking that all ranks carry the same record 1;
 * dasha_restart_write_ranks splits a global state into the rank files, each local entry taken
 * from the global node it stands for (x periodic, zeros beyond the z walls), which readin
 * then refreshes between ranks (message4).  Records as in dasha_restart_write. */
int dasha_restart_read_ranks(const char* dir, int nst_file, int nprx, int nprz, int* ncase, int* nstep, double* time,
                             int* nst, int mx, int my, int mz, double* x_f, long ld1, long ld2);
int dasha_restart_write_ranks(const char* dir, int ncase, int nstep, double time, int nst, int nprx, int nprz, int mx,
                              int my, int mz, const double* x_f, long ld1, long ld2, long max_subrecord);

/* ASCII mid-plane file m2dNNN.dat of recrd2 (t3dsdsc.f:5116-5154): list-directed lines
 * "2 mx mz" and time, the coordinates x[mx] then z[mz] as one list, then for q = 1..11 a line
 * "q" and plane field q-1 (the layout dasha_midplane returns), all lists in the format
 * 5(1X,E14.5E3). */
int dasha_m2d_write(const char* path, int mx, int mz, double time, const double* x, const double* z,
                    const double* plane);

/* The same eleven fields as dasha_midplane, gathered on the host from a state array and a
 * current array in the dasha_get_state / dasha_current layout. */
int dasha_midplane_host(int mx, int my, int mz, const double* x_f, const double* cur_f, long ld1, long ld2,
                        double* plane);

/* ASCII 3-D file m3dNNN of recrd3 (t3dsdsc.f:5365-5402): "3 mx my mz", time, x, y, z as one
 * list, then for q = 1..11 a line "q" and field q on all nodes (x fastest, then y, then z),
 * the fields of dasha_midplane formed from the state x_f and the current cur_f (layouts of
 * dasha_get_state / dasha_current), all lists in the format 11(1X,E10.4). */
int dasha_m3d_write(const char* path, int mx, int my, int mz, double time, const double* x, const double* y,
                    const double* z, const double* x_f, const double* cur_f, long ld1, long ld2);

/* One line of current.dat, the file diagn writes every 10 steps (t3dsdsc.f:1226-1232): the
 * mid-y-plane current extrema diag[3..8] of dasha_diagnostics (Jx max, Jx min, Jy max, Jy min,
 * Jz max, Jz min) and time, in the format 7(1X,E13.4).  append = 0 starts the file (the first
 * call of a run), 1 adds the line at its end. */
int dasha_current_dat_write(const char* path, const double* diag, double time, int append);

/* The main loop's step logs (t3dsdsc.f:157-181), each call appending one line:
 * dasha_stepnm_write: ./data/stepnm, "nstep time dt" before the step (list-directed; integers in
 * 12 columns, reals with 17 significant digits); dasha_dtlog_write: unit 20 (fort.20), dt, time
 * and nstep after the step in the format 2(1X,F10.5),1X,I5. */
int dasha_stepnm_write(const char* path, int nstep, double time, double dt);
int dasha_dtlog_write(const char* path, double dt, double time, int nstep);

const char* dasha_last_error(dasha_ctx* ctx);
void dasha_destroy(dasha_ctx* ctx);

#ifdef __cplusplus
}
#endif
#endif
