/*
 * dgbgk.h -- C ABI of the B200 (sm_100a) implementation of the DG-BGK
 * transport-plus-collision pseudo-time sweep.
 *
 * The library replaces the reference time step ADVNCE (src/advnce.f90:3-25,
 * called once from src/dg_lin_convec.f90:185-206) and the output gather
 * GETMAC (src/getmac.f90:3-127).  A host written in any language binds these
 * entry points; a Fortran host binds them through ISO_C_BINDING interfaces
 * with the same argument lists (BIND(C), VALUE for the scalars).
 *
 * Conventions
 *  - Every array argument is caller-owned host memory and is copied in or
 *    out; the library owns all device memory.  No torch or CUDA types appear
 *    in the signatures.
 *  - Mesh arrays keep the reference's Fortran layout: column-major with the
 *    reference's leading dimensions, 1-based node/element indices
 *    (INTMA(3,NELEM), BSIDO(6,NBOUN), ISIDE(8,NSIDE) ...).  Reals are double.
 *  - The distribution function keeps the reference layout
 *    DISNF(3, VNPNT, NELEM), column-major (src/dg_lin_convec.f90:93).
 *  - Status: 0 = success; a negative DGBGK_E* code otherwise, with a message
 *    from dgbgk_last_error().  The library never calls exit().
 *  - One host thread per handle; distinct handles may be used from distinct
 *    threads.
 */
#ifndef DGBGK_H
#define DGBGK_H

#ifdef __cplusplus
extern "C" {
#endif

#define DGBGK_OK 0
#define DGBGK_EINVAL (-1)    /* bad size, pointer or parameter */
#define DGBGK_EMESH (-2)     /* inconsistent mesh (node out of range, side or wall not found, zero area or length) */
#define DGBGK_ECUDA (-3)     /* CUDA runtime error or no usable sm_100 GPU */
#define DGBGK_ENONFINITE (-4) /* non-finite residual: the state diverged */
#define DGBGK_EUNSUP (-5)    /* configuration not supported by this build */

typedef struct dgbgk_handle dgbgk_handle;

/* Mesh and the geometric arrays the reference computes during setup
 * (src/dg_lin_convec.f90:96-125): GETSID, NORMAL, GETGEO, GETLEN,
 * GETMAT/CONMAT, GETNOR.  dgbgk_setup_mesh() below computes them from
 * INTMA, COORD and BSIDO the same way. */
typedef struct dgbgk_mesh {
  int nelem, npoin, nboun, nside;
  const int* intma;     /* INTMA(3,NELEM)            src/gtinpt.f90:27-29  */
  const double* coord;  /* COORD(2,NPOIN)            src/gtinpt.f90:36-38  */
  const int* bsido;     /* BSIDO(6,NBOUN)            src/gtinpt.f90:48-50  */
  const int* iside;     /* ISIDE(8,NSIDE)            src/getsid.f90:1-216 */
  const double* nx;     /* NX(NSIDE)                 src/normal.f90:24-33  */
  const double* ny;     /* NY(NSIDE)                                       */
  const double* el;     /* EL(NSIDE)                                       */
  const double* geome;  /* GEOME(7,NELEM)            src/getgeo.f90:22-59  */
  const double* relen;  /* RELEN(NELEM)              src/getlen.f90:17-26  */
  const double* mmat;   /* MMAT(3,NELEM), IMMAT = 1  src/getmat.f90:17-40  */
  const double* cmmat;  /* CMMAT(3,3,NELEM), IMMAT=0 src/conmat.f90:17-41  */
  const double* rsido;  /* RSIDO(3,NBOUN)            src/getnor.f90:21-31  */
} dgbgk_mesh;

/* Velocity space: VCORD(3,VNPNT) and SUMWEIGHT from VSPACE
 * (src/vspace.f90:16-50); rv = IVD%rv. */
typedef struct dgbgk_vspace {
  int rorder, torder;
  const double* vcord;
  double sumweight;
  double rv;
} dgbgk_vspace;

/* Physical and numerical parameters (the namelist of
 * src/input_variable_module.f90:4-34 as ADVNCE receives them). */
typedef struct dgbgk_params {
  int immat;          /* 1: lumped mass (GETINC), 0: consistent (CMMINC)  */
  double csafm;       /* Courant safety factor                            */
  double alpha;       /* wall accommodation (1 = fully diffuse; < 1 adds the
                         specular part, with either immat)                 */
  double rgas;        /* gas constant R                                   */
  double molar_mass;  /* M                                                */
  double diameter;    /* molecular diameter d                             */
  double cinf[4];     /* inflow T, P [bar], U, V (zeros when IVD%INF = 0) */
  /* Extensions: each reduces to the reference when left at its default.  */
  int precision;      /* 64 (default): f in FP64; 32: f stored and swept
                         in FP32 with FP64 moments and residual norms      */
  const double* wall_velocity; /* (2,NBOUN) moving-wall velocity per
                                  boundary side, or NULL (all at rest)    */
  int tile_elems;     /* sweep tile: elements per CTA, 64 or 128 (0: 128 for FP32, 64 for FP64) */
  int moment_rows;    /* moment kernel: velocity rows per warp step -- 1, 2 or 4
                         rows of any elements (32/R lanes per row), or 3: the
                         three rows of one element on all 32 lanes (0 = the
                         library's choice) */
  int device;         /* CUDA device ordinal                               */
  int shard;          /* 1: the handle holds a velocity shard -- the vspace
                         passed has only its speed rings (RORDER = their
                         count), with the full grid's SUMWEIGHT -- and its
                         steps run through dgbgk_shard_* (0 = whole grid) */
} dgbgk_params;

/* Fills a dgbgk_params with the reference defaults of
 * src/spectralbgk.f90:116-147 plus precision 64. */
void dgbgk_default_params(dgbgk_params* p);

/* Host-side setup: GETSID (src/getsid.f90:1-216), NORMAL
 * (src/normal.f90:24-33), GETGEO (src/getgeo.f90:22-59), GETLEN
 * (src/getlen.f90:17-26), GETMAT (src/getmat.f90:17-40) or CONMAT
 * (src/conmat.f90:17-41) and GETNOR (src/getnor.f90:21-31) from INTMA, COORD
 * and BSIDO.  Output capacities: iside 8*mxsid, nx/ny/el mxsid with
 * mxsid = 2*(nelem+nboun) (src/spectralbgk.f90:274); geome 7*nelem; relen
 * nelem; mmat 3*nelem; cmmat 9*nelem; rsido 3*nboun.  *nside receives NSIDE. */
int dgbgk_setup_mesh(int nelem, int npoin, int nboun, const int* intma, const double* coord,
                     const int* bsido, int* nside, int* iside, double* nx, double* ny, double* el,
                     double* geome, double* relen, double* mmat, double* cmmat, double* rsido);

/* Velocity grid: VSPACE (src/vspace.f90:16-50) from the Lobatto pairs
 * (eta_i, w_i), i = 1..rorder, with torder uniform angles.  vcord gets
 * 3*rorder*torder values. */
int dgbgk_vspace_build(int rorder, int torder, const double* eta, const double* w, double* vcord,
                       double* sumweight);

/* Creates a solver on the GPU; copies every input.  Replaces the setup part
 * of ADVNCE (src/advnce.f90:127-148, ALOTIM and the first MACROS). */
int dgbgk_create(const dgbgk_mesh* mesh, const dgbgk_vspace* vs, const dgbgk_params* prm,
                 dgbgk_handle** out);

/* State transfer in the reference layout DISNF(3,VNPNT,NELEM). */
int dgbgk_set_state(dgbgk_handle* h, const double* disnf);
int dgbgk_get_state(dgbgk_handle* h, double* disnf);
int dgbgk_set_state_f32(dgbgk_handle* h, const float* disnf);
int dgbgk_get_state_f32(dgbgk_handle* h, float* disnf);

/* INICON2 (src/inicon2.f90:116-180): the uniform Maxwellian at T1, P1 [bar],
 * (U0, V0), optionally scaled per DG node by node_scale(3,NELEM) (NULL = 1;
 * the seeded density perturbation of the benchmark cases).  Built on the
 * device. */
int dgbgk_init_uniform(dgbgk_handle* h, double t1, double p1, double u0, double v0,
                       const double* node_scale);

/* Maxwellian per DG node from nodal fields (the warm start): number
 * density n, velocity (u, v) and temperature T, each (3,NELEM) per DG node,
 * with the INICON2 formula. */
int dgbgk_init_maxwellian(dgbgk_handle* h, const double* n, const double* u, const double* v,
                          const double* t);

/* The ADVNCE time loop (src/advnce.f90:220-449): runs steps until max_steps
 * have run or the L2 residual falls to tol_rel times the reference residual
 * (tol_rel <= 0: run all max_steps).  The reference residual is the L2
 * residual of the first step this handle ever ran unless set with
 * dgbgk_set_residual_reference().  Per step, when non-NULL, res_linf gets
 * max|DELUN| (the value behind RESIDUAL.RES, src/advnce.f90:422-429),
 * res_l2 the L2 norm of the change the unknowns receive (DELUN, -f where
 * ADTHEM clips, nothing at the DG nodes INFLOW resets) and dte the time
 * step.  *steps_done gets the number of steps run. */
int dgbgk_advance(dgbgk_handle* h, int max_steps, double tol_rel, int* steps_done, double* res_linf,
                  double* res_l2, double* dte);
int dgbgk_set_residual_reference(dgbgk_handle* h, double res_l2_ref);
int dgbgk_get_residual_reference(dgbgk_handle* h, double* res_l2_ref);

/* No counterpart in the reference.  Copies the state of `src` into `dst`
 * on the device, converting between the handles' precisions (FP32 <-> FP64),
 * and hands over the residual reference: the precision handoff of a march
 * that runs its transient in FP32 and finishes in FP64.  Both handles must
 * be on one device and built from the same mesh and velocity grid. */
int dgbgk_copy_state(dgbgk_handle* dst, const dgbgk_handle* src);


/* No counterpart in the reference.  Reduced-rank extrapolation of the
 * pseudo-time iterates, a way to reach the same fixed point in fewer steps:
 * dgbgk_snapshot copies the current state into slot (0 <= slot < 11; the
 * slots' device storage grows as they are first used, doubling up to 11;
 * slot < 0 frees them).  dgbgk_extrapolate takes the snapshots x_0 .. x_{n-1} of
 * consecutive iterates, finds gamma (n-1 values, sum 1) minimising
 * |sum_j gamma_j (x_{j+1} - x_j)|, and replaces the state by
 * max(sum_j gamma_j x_j, 0); gamma (may be NULL) receives the coefficients.
 * The march goes on from there: its residual test decides convergence as
 * before. */
int dgbgk_snapshot(dgbgk_handle* h, int slot);
int dgbgk_extrapolate(dgbgk_handle* h, int n, double* gamma);

/* GETFOR (src/getfor.f90:29-49) of the current state: the lift and drag
 * of the type-4 wall sides from the nodal pressure, reduced on the device
 * after MACROS + GETMAC; two numbers cross to the host. */
int dgbgk_get_forces(dgbgk_handle* h, double* lift, double* drag);

/* ADVNCE's periodic output (src/advnce.f90:403-417, GETFOR at :427-435)
 * without a host round trip: with every > 0, dgbgk_advance records GETMAC's
 * nodal fields (ND, RHO, UVEL, VVEL, PS, TEMP) and GETFOR's lift and drag
 * whenever ITIME -- the steps the handle has run since its state was last
 * set (dgbgk_set_state*, dgbgk_init_*), counted across advance calls and
 * carried over by dgbgk_copy_state -- is a multiple of `every`, into a
 * device ring of `capacity` records (the oldest is overwritten).  Each call
 * replaces the ring; every = 0 stops recording.  Batches do not record. */
int dgbgk_set_output(dgbgk_handle* h, int every, int capacity);
/* Records taken since dgbgk_set_output (the ring holds the last
 * min(count, capacity)). */
int dgbgk_output_count(dgbgk_handle* h, int* count);
/* Record k of those held (0 = the oldest): its ITIME, the six nodal fields
 * (NPOIN values each) and lift and drag; any pointer may be NULL. */
int dgbgk_get_output(dgbgk_handle* h, int k, int* itime, double* nd, double* rho, double* u, double* v, double* ps,
                     double* temp, double* lift, double* drag);

/* MACROS (src/macros.f90:51-188) + GETMAC (src/getmac.f90:98-123) of the
 * current state: nodal ND, RHO, UVEL, VVEL, PS, TEMP, NPOIN values each. */
int dgbgk_get_macros(dgbgk_handle* h, double* nd, double* rho, double* u, double* v, double* ps,
                     double* temp);

/* Discontinuous per-DG-node fields of the current state (each (3,NELEM)):
 * DISND, DISUX, DISUY, DISPS (src/macros.f90:131-164) and MU
 * (src/compmu.f90:86-97).  Any pointer may be NULL. */
int dgbgk_get_node_fields(dgbgk_handle* h, double* disnd, double* disux, double* disuy,
                          double* disps, double* mu);

/* FLUCON2 (src/flucon2.f90:43-241) of the current state: ETA(NBOUN). */
int dgbgk_get_wall_eta(dgbgk_handle* h, double* eta);

/* Sizes: [NELEM, NPOIN, NBOUN, NSIDE, VNPNT, precision, tile_elems,
 * tile_vels, n_blocks, max_halo]. */
int dgbgk_info(dgbgk_handle* h, int* out10);

/* Device time of the last dgbgk_advance() call in ms (CUDA events on the
 * library's stream around the whole time loop). */
int dgbgk_last_timing(dgbgk_handle* h, double* total_ms);

/* Runs nsteps time steps launch by launch (no graph) with CUDA events
 * between the kernels on the library's stream; kernel_ms[4] receives the
 * mean device time per step of [moments, wall flux, sweep, residual]. The
 * state advances by nsteps steps exactly as under dgbgk_advance(). */
int dgbgk_profile_steps(dgbgk_handle* h, int nsteps, double* kernel_ms);

/* No counterpart in the reference.  dgbgk_get_macros() without any device
 * allocation, for callers that cannot allocate GPU memory at call time: a
 * host whose device memory is owned by another allocator or pool, a time
 * loop that must not pay the device-wide synchronisation of cudaMalloc /
 * cudaFree while other streams run, or code that runs after its memory
 * budget is fixed.  The nodal fields are staged in one static device array
 * of 6*DGBGK_NOALLOC_MAX_NPOIN doubles (~6.3 MB) that every GPU loading the
 * library holds until the process exits; meshes with NPOIN above the limit
 * are rejected with DGBGK_EINVAL.  The first call on a device takes the
 * array's device address (cudaGetSymbolAddress) and should come before any
 * stream capture.  All calls share the one array: calls that overlap on the
 * GPU (from several handles or threads on the same device) race and must
 * be serialised by the caller. */
#define DGBGK_NOALLOC_MAX_NPOIN 131072
int dgbgk_get_macros_noalloc(dgbgk_handle* h, double* nd, double* rho, double* u, double* v, double* ps,
                             double* temp);

/* ---- Velocity-space shards ----------------------------------------------
 * The reference splits velocity space into NVSPACEPART blocks of whole speed
 * rings (src/spectralbgk.f90:163-199) and sums the partial velocity sums of
 * MACROS, COMPMU and FLUCON2 over them with MPI_ALLREDUCE
 * (src/macros.f90:114-119, 153-154; src/compmu.f90:80-81;
 * src/flucon2.f90:215-216).  A handle created with dgbgk_params.shard = 1
 * and a vspace of its rings only (RORDER = the rings' count, VCORD their
 * rows, SUMWEIGHT the full grid's; ALPHA = 1) is such a block.  Its step
 * runs in phases on the handle's stream; between them the caller sums the
 * exchange buffers over the shards (device memory the caller owns, of the
 * sizes dgbgk_shard_sizes gives) -- an NCCL all-reduce enqueued on that
 * stream, for one shard per GPU:
 *   phase 1: pass-1 partial sums            -> sums1        (then SUM)
 *   phase 2: pass-2 partial sums and walls  -> sums2        (then SUM)
 *   phase 3: moments, MU, dt, ETA; the sweep of the shard's velocities;
 *            the step's residual partials    -> res[2]      (then MAX of
 *            res[0], SUM of res[1])
 *   phase 4: the step's bookkeeping (histories, convergence test).
 * dgbgk_shard_begin / _end bracket a run of steps as dgbgk_advance does
 * (its max_steps, tol, histories and status); phases 0 (outside a run),
 * 1, 2 and 5 give dgbgk_get_macros, _get_forces and _get_node_fields the
 * moments of the current state.  dgbgk_advance, batches and the output ring
 * refuse a shard. */
int dgbgk_shard_stream(dgbgk_handle* h, void** stream);  /* the cudaStream_t of the phases */
int dgbgk_shard_sizes(dgbgk_handle* h, long long* n_sums1, long long* n_sums2);  /* doubles */
int dgbgk_shard_begin(dgbgk_handle* h, int max_steps, double tol);
int dgbgk_shard_phase(dgbgk_handle* h, int phase, double* sums1, double* sums2, double* res);
int dgbgk_shard_poll(dgbgk_handle* h, int* done);  /* synchronises the stream */
int dgbgk_shard_end(dgbgk_handle* h, int* steps_done, double* res_linf, double* res_l2, double* dte, int* done);

void dgbgk_destroy(dgbgk_handle* h);
const char* dgbgk_last_error(void);

/* ---- Batches (no counterpart in the reference) --------------------------
 * Many cases -- handles of the same precision, IMMAT and device, each with
 * its own mesh, velocity grid and state -- advanced together: every kernel
 * of a pseudo-time step is one persistent launch over the flattened work of
 * all the cases, and steps are replayed from one CUDA graph.  Each case
 * keeps its own time step, residual history, reference and convergence
 * test; cases that converge (or reach max_steps) stop while the others go
 * on.  The handles stay usable on their own between batch calls (not
 * concurrently with them). */
typedef struct dgbgk_batch dgbgk_batch;

typedef struct {
  int tile_elems;     /* sweep elements per CTA, 64 or 128 (0: autotuned)    */
  int units_per_cta;  /* sweep work units per resident CTA, 2/4/8/16 (0: autotuned) */
  int tune_steps;     /* steps timed per autotuner candidate                */
  int moment_rows;    /* moment rows per warp step, 1/2/3/4 (0: autotuned)   */
} dgbgk_batch_params;

void dgbgk_batch_default_params(dgbgk_batch_params* p);

/* Creates a batch over `ncases` handles.  The autotuner times every
 * candidate tile shape (elements per CTA x units per CTA) on the cases'
 * current states for `tune_steps` steps, restores the states, and keeps
 * the fastest. */
int dgbgk_batch_create(dgbgk_handle* const* cases, int ncases, const dgbgk_batch_params* p,
                       dgbgk_batch** out);

/* Advances every active case until its L2 residual falls to tol times its
 * reference (tol <= 0: no test) or it has run max_steps steps.
 * steps_done[ncases] and res_l2_last[ncases] (either may be NULL) receive
 * each case's step count and last L2 residual (0 steps and 0.0 for a case
 * that did not run); the per-step histories stay in the handles' devices
 * and are not returned here.  A case that diverged (DGBGK_ENONFINITE) or
 * whose device wait expired stays stopped, with that status, in later
 * advances until its state is set again (dgbgk_set_state*, dgbgk_init_*,
 * dgbgk_copy_state, dgbgk_extrapolate).  If a handle was changed on its own
 * in a way that moved its device buffers (a longer dgbgk_advance, another
 * batch's tile shape), the batch rebuilds its case table first. */
int dgbgk_batch_advance(dgbgk_batch* b, int max_steps, double tol, int* steps_done, double* res_l2_last);

/* active[ncases]: 0 leaves case i out of the following advances (0 steps,
 * its state untouched), non-zero takes it back; every case starts active. */
int dgbgk_batch_set_active(dgbgk_batch* b, const int* active);

/* status[ncases]: each case's result of the last dgbgk_batch_advance()
 * (DGBGK_OK, DGBGK_ENONFINITE for a case that diverged and stopped, ...);
 * the advance itself returns the first non-zero one. */
int dgbgk_batch_status(const dgbgk_batch* b, int* status);

/* [ncases, tile_elems, units_per_cta, sweep work units, sweep CTAs,
 * moment CTAs, moment rows per warp step] of the chosen configuration. */
int dgbgk_batch_info(const dgbgk_batch* b, int* out7);

/* The autotuner's ms per batch step: (tile_elems 64, 128) x (units_per_cta
 * 2, 4, 8, 16), then moment rows per warp step 1, 2, 3, 4 at the chosen
 * sweep shape; 0 where not tried; n <= 12. */
int dgbgk_batch_tuning(const dgbgk_batch* b, int n, double* ms_per_step);

/* Device time of the last dgbgk_batch_advance() in ms. */
int dgbgk_batch_last_timing(const dgbgk_batch* b, double* total_ms);

/* No counterpart in the reference.  dgbgk_snapshot(case, slot) of every
 * case with which[i] non-zero (which may be NULL: all cases), the copies
 * queued on the batch's stream without a wait; the next advance and every
 * later use of a case follow them. */
int dgbgk_batch_snapshot(dgbgk_batch* b, int slot, const int* which);

/* dgbgk_extrapolate(case, n, ...) of every case with which[i] non-zero
 * (NULL: all), the Gram matrices of all of them formed before one wait.
 * status[ncases] receives each case's result (DGBGK_OK, or the code
 * dgbgk_extrapolate would return; 0 for cases not selected; a case that
 * fails keeps its state), gamma (may be NULL) n-1 coefficients per case at
 * gamma[i*(n-1)].  Returns the first non-zero status. */
int dgbgk_batch_extrapolate(dgbgk_batch* b, int n, const int* which, int* status, double* gamma);

void dgbgk_batch_destroy(dgbgk_batch* b);

/* ---- Warm-start network (no counterpart in the reference) ---------------
 * A multilayer perceptron n_in -> width x depth (tanh) -> n_out trained and
 * evaluated with hand-written BF16 tensor-core kernels (tcgen05, FP32
 * accumulation in tensor memory, FP32 master weights, Adam).  It maps case
 * parameters to resampled steady fields whose Maxwellian starts the solver
 * (dgbgk_init_maxwellian).  Sizes: n_in <= 64; width, n_out and batch
 * multiples of 128. */
typedef struct dgbgk_mlp dgbgk_mlp;

int dgbgk_mlp_create(int n_in, int width, int depth, int n_out, int batch, unsigned long long seed, int device,
                     dgbgk_mlp** out);
/* Number of parameters; per layer W[out][in] (the input layer's in is 64,
 * columns past n_in zero) then b[out], layers in order. */
long long dgbgk_mlp_param_count(const dgbgk_mlp* m);
int dgbgk_mlp_get_params(dgbgk_mlp* m, float* params);
int dgbgk_mlp_set_params(dgbgk_mlp* m, const float* params);
/* y[n][n_out] = network(x[n][n_in]) */
int dgbgk_mlp_forward(dgbgk_mlp* m, const float* x, int n, float* y);
/* Mean squared error and its gradient (the parameter layout) on one batch
 * of exactly `batch` rows. */
int dgbgk_mlp_gradient(dgbgk_mlp* m, const float* x, const float* t, int n, double* loss, float* grad);
/* Training set x[n][n_in], t[n][n_out], kept on the device. */
int dgbgk_mlp_set_data(dgbgk_mlp* m, const float* x, const float* t, int n);
/* iters Adam steps (learning rate lr) on minibatches drawn without
 * replacement per epoch (seeded); loss_hist[iters] may be NULL. */
int dgbgk_mlp_train(dgbgk_mlp* m, int iters, float lr, unsigned long long seed, double* loss_hist);
void dgbgk_mlp_destroy(dgbgk_mlp* m);

#ifdef __cplusplus
}
#endif
#endif /* DGBGK_H */
