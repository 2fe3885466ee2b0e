/*
 * cgfd.h -- C ABI of the B200 dynamic-rupture solver (libcgfd.so).
 *
 * The reference exposes no library interface: its whole forward path sits
 * behind one host function,
 *
 *   int drv_rk_curv_col_allstep(fd_t*, gd_t*, gd_metric_t*, md_t*, par_t*,
 *        bdryfree_t*, bdrypml_t*, bdryexp_t*, wav_t*, mympi_t*,
 *        fault_coef_t*, fault_t*, fault_wav_t*, iorecv_t*, ioline_t*,
 *        iofault_t*, ioslice_t*, iosnap_t*, io_fault_recv_t*,
 *        float dt, int nt_total, float t0, char*, char*)
 *   (src/forward/drv_rk_curv_col.cu:29-52, called from
 *    src/forward/main_curv_col_el_3d.cu:711)
 *
 * preceded by host set-up (grid, metric, medium, PML, fault coefficients;
 * main_curv_col_el_3d.cu:113-705).  This header replaces both with a
 * handle: cgfd_create() takes the same inputs as plain host arrays, does the
 * set-up and copies everything to the GPU once; cgfd_run() advances the
 * forward time loop; the getters read back the fault fields, the station
 * seismograms and the wavefield.
 *
 * Axes are the reference's: x (index i) is the fault-normal direction, y
 * (index j) is along strike, z (index k) points up and the free surface is
 * the top plane k = nk-1.  Every array is C order with x fastest:
 * 3-D arrays are [nk][nj][ni], fault-plane arrays are [nk][nj].
 *
 * Conventions: every call returns CGFD_OK (0) or a negative CGFD_ERR_*
 * code and never exits the process; cgfd_last_error() returns a message for
 * the last failing call of the calling thread.  A handle may be used by one
 * host thread at a time.  The caller owns every pointer it passes; the
 * library copies what it needs during cgfd_create().
 */
#ifndef CGFD_H
#define CGFD_H

#ifdef __cplusplus
extern "C" {
#endif

#define CGFD_ABI_VERSION 2

#define CGFD_MAX_FAULTS 8

/* status codes */
#define CGFD_OK              0
#define CGFD_ERR_ARG        -1   /* invalid argument or configuration      */
#define CGFD_ERR_CUDA       -2   /* CUDA runtime error                     */
#define CGFD_ERR_NOMEM      -3   /* device or host allocation failed       */
#define CGFD_ERR_UNSTABLE   -4   /* NaN/Inf found in the wavefield         */
#define CGFD_ERR_DT         -5   /* dt above the CFL limit of the grid     */
#define CGFD_ERR_NODEVICE   -6   /* no CUDA device / kernels not loadable  */
#define CGFD_ERR_STATE      -7   /* call not valid in the handle's state   */

/* grid generation (par key "grid_generation_method") */
#define CGFD_GRID_FAULT_PLANE 0  /* extrude fault surfaces along x        */
#define CGFD_GRID_IMPORT      1  /* caller gives all (x,y,z) coordinates  */

/* fault output fields, order of the reference's fault_t.output
 * (src/forward/fault_info.cu:865-942) */
#define CGFD_FAULT_TN      0
#define CGFD_FAULT_TS1     1
#define CGFD_FAULT_TS2     2
#define CGFD_FAULT_VS      3
#define CGFD_FAULT_VS1     4
#define CGFD_FAULT_VS2     5
#define CGFD_FAULT_SLIP    6
#define CGFD_FAULT_SLIP1   7
#define CGFD_FAULT_SLIP2   8
#define CGFD_FAULT_PEAK_VS 9
#define CGFD_FAULT_INIT_T0 10
#define CGFD_FAULT_NFIELD  11

/* wavefield components, order of the reference's wav_t
 * (src/forward/wav_t.cu:57-108) */
#define CGFD_VX  0
#define CGFD_VY  1
#define CGFD_VZ  2
#define CGFD_TXX 3
#define CGFD_TYY 4
#define CGFD_TZZ 5
#define CGFD_TYZ 6
#define CGFD_TXZ 7
#define CGFD_TXY 8
#define CGFD_NCMP 9

typedef struct cgfd_config {
  /* interior grid points ("number_of_total_grid_points_{x,y,z}") */
  int ni, nj, nk;
  /* time step ("size_of_time_step"); checked against the CFL limit
   * (CFL 1.3, src/forward/fd_t.cu:57) unless check_stability == 0 */
  float dt;
  int check_stability;
  /* "dynamic_method": 1 (continuity matrices) or 2 (traction rate) */
  int dynamic_method;
  /* faults: constant-x planes; indices are 1-based as in the par file */
  int num_faults;
  int fault_x_index[CGFD_MAX_FAULTS];     /* "fault_x_index"           */
  int fault_grid[CGFD_MAX_FAULTS][4];     /* "fault_grid" j1,j2,k1,k2  */
  /* nodes closer than this to the y sides (and to the bottom, or to the
   * top without free surface) are welded; the reference hard-codes 40
   * (src/forward/fault_info.cu:1044-1060) */
  int welded_margin;
  /* 1: traction-image free surface on the top face ("boundary_z_top":
   * {"free": ...}) */
  int free_surface;
  /* CFS-PML per face [dim x,y,z][side left/bottom, right/top]; 0 layers =
   * no PML ("boundary_*": {"cfspml": {...}}) */
  int   pml_layers[3][2];
  float pml_alpha_max[3][2];
  float pml_beta_max[3][2];
  float pml_ref_vel[3][2];
  /* geometry */
  int grid_mode;                 /* CGFD_GRID_FAULT_PLANE / CGFD_GRID_IMPORT */
  float fault_interval;          /* "fault_inteval": x spacing (FAULT_PLANE) */
  const float *fault_x, *fault_y, *fault_z;   /* [num_faults][nk][nj]        */
  const float *x3d, *y3d, *z3d;               /* [nk][nj][ni] (GRID_IMPORT)   */
  /* isotropic elastic medium, [nk][nj][ni] */
  const float *lambda, *mu, *rho;
  /* fault initial traction and friction ("init_stress_<id>.nc"),
   * [num_faults][nk][nj] */
  const float *T0x, *T0y, *T0z, *mu_s, *mu_d, *Dc, *C0;
  /* volume stations: 0-based global interior grid index (i, j, k),
   * fractional parts interpolate; [num_stations][3] */
  int num_stations;
  const float *station_ijk;
  /* fault stations: fault id (0-based) and 0-based (j, k) on the fault
   * plane, fractional parts interpolate; [num_fault_stations] and [..][2] */
  int num_fault_stations;
  const int   *fault_station_fault;
  const float *fault_station_jk;
  /* capacity of the station/fault-station time series (records) */
  int max_records;
  /* exponential sponge per face [dim][side] ("boundary_*": {"ablexp":
   * {"number_of_layers", "ref_vel"}}): every step the end-of-step level is
   * multiplied by exp(-alpha (n/L)^2) in the outer L layers
   * (bdry_ablexp_set / bdry_ablexp_apply, src/forward/bdry_t.cu:453-818).
   * 0 layers = no sponge.  Sponge faces cannot be combined with cfspml
   * faces (the reference then computes masks for the PML faces from an
   * unset velocity), nor with the free top. */
  int   ablexp_layers[3][2];
  float ablexp_ref_vel[3][2];
} cgfd_config;

typedef struct cgfd_solver cgfd_solver;
typedef struct cgfd_setup cgfd_setup;

/* ABI version compiled into the library (CGFD_ABI_VERSION). */
int cgfd_abi_version(void);

/* Host half of cgfd_create: grid, metric, medium, PML, free-surface and
 * fault set-up into host memory (main_curv_col_el_3d.cu:113-705).  Needs
 * no GPU; when a device is present, the packed metric and medium are kept
 * in page-locked host memory so that cgfd_upload copies them at link rate
 * (this initialises the CUDA context of the current device). */
int cgfd_prepare(const cgfd_config *cfg, cgfd_setup **out);
/* Bytes that cgfd_upload copies to the device. */
int cgfd_setup_bytes(const cgfd_setup *su, unsigned long long *bytes);
/* Grid coordinates of a prepared problem, interior points, [nk][nj][ni]
 * each (any of x, y, z may be NULL): the imported grid, or the grid the
 * fault-plane extrusion made (gd_curv_gen_fault, gd_t.cu:402-545). */
int cgfd_setup_coords(const cgfd_setup *su, float *x, float *y, float *z);
/* Largest stable dt of a prepared problem (CFL 1.3). */
int cgfd_setup_dt_max(const cgfd_setup *su, float *dtmax);
/* Device half of cgfd_create: allocate the device state on the current
 * device and copy the prepared problem (drv_rk_curv_col.cu:90-100). */
int cgfd_upload(const cgfd_setup *su, cgfd_solver **out);
void cgfd_setup_free(cgfd_setup *su);

/* Make GPU `ordinal` the current device of the calling thread for the
 * calls that follow (the reference's gpu_id_start argument of main). */
int cgfd_select_device(int ordinal);

/* Device memory of solvers comes from the current device's stream-ordered
 * memory pool, which keeps the blocks of destroyed solvers for the next
 * ones (no counterpart in the reference, which calls cudaMalloc / cudaFree
 * around each run).  This returns the cached blocks of the current device
 * to the system, after waiting for the device to be idle. */
int cgfd_release_cached_memory(void);

/* Fill cfg with the reference's defaults (welded margin 40, dynamic
 * method 2, stability check on, no PML, free surface off). */
void cgfd_config_default(cgfd_config *cfg);

/* Set up grid, metric, medium, PML and fault coefficients on the host and
 * move the problem to the current CUDA device.
 * Replaces main_curv_col_el_3d.cu:113-705 + the device set-up at
 * drv_rk_curv_col.cu:90-100. */
int cgfd_create(const cgfd_config *cfg, cgfd_solver **out);

/* Advance nsteps time steps (4 RK stages each); before each step the
 * stations and fault stations are sampled, as io_recv_keep /
 * io_fault_recv_keep do at drv_rk_curv_col.cu:215-218.
 * Replaces the time loop of drv_rk_curv_col.cu:209-636. */
int cgfd_run(cgfd_solver *s, int nsteps);

/* Advance nsteps time steps like cgfd_run and take the fault output the
 * reference writes while it steps: before every step whose index (steps
 * taken so far) is a multiple of `every` (io_time_skip), the 11 fault
 * fields of every fault, interior nodes, go to
 * out[record][fault][11][nk][nj] (the data of io_fault_nc_put,
 * src/forward/io_funcs.cu:2027-2099, called at drv_rk_curv_col.cu:221-226).
 * Each record is gathered on the device into one of two staging buffers
 * and copied on a separate stream while the next steps run; with `out` in
 * page-locked memory the copies overlap the stepping.  `max_records`: the
 * records `out` holds; a run that would take more is rejected with
 * CGFD_ERR_ARG before anything runs.  *nrec: the records taken (may be
 * NULL).  No counterpart as a function in the reference, whose loop blocks
 * on each output copy. */
int cgfd_run_fault_output(cgfd_solver *s, int nsteps, int every, float *out, long long max_records, int *nrec);

/* Page-locked host memory for the output buffers of cgfd_run_fault_output
 * (and any getter), for callers that do not link the CUDA runtime
 * themselves; free it with cgfd_host_free.  No reference counterpart. */
int cgfd_host_alloc(unsigned long long bytes, void **ptr);
void cgfd_host_free(void *ptr);

/* Number of steps taken so far. */
int cgfd_steps_done(const cgfd_solver *s, int *it);

/* Dense grid spacing bound: largest dt that passes the stability check. */
int cgfd_dt_max(const cgfd_solver *s, float *dtmax);

/* One fault field (CGFD_FAULT_*) of fault `fault_id` (0-based), interior
 * nodes, [nk][nj].  The data behind io_fault_nc_put
 * (src/forward/io_funcs.cu:2027-2099). */
int cgfd_get_fault(cgfd_solver *s, int fault_id, int field, float *out);

/* All 11 fault fields of one fault at once, [11][nk][nj]. */
int cgfd_get_fault_all(cgfd_solver *s, int fault_id, float *out);

/* Station seismograms [num_stations][9][nrec], nrec = records taken so
 * far (*nrec set on return, <= max_records). */
int cgfd_get_stations(cgfd_solver *s, float *out, int *nrec);

/* Fault-station time series [num_fault_stations][9][nrec] of
 * Tn,Ts1,Ts2,Vs,Vs1,Vs2,Slip,Slip1,Slip2. */
int cgfd_get_fault_stations(cgfd_solver *s, float *out, int *nrec);

/* Peak ground motion of the free surface over the steps run so far
 * (PG_calcu_gpu, src/forward/wav_t.cu:138-216): [CGFD_NPEAK][nj][ni] in the
 * order PGV, PGVh, PGVx, PGVy, PGVz, PGA, PGAh, PGAx, PGAy, PGAz, PGD, PGDh,
 * PGDx, PGDy, PGDz (the variables of PG_V_A_D_*.nc, io_funcs.cu:1827-1880).
 * CGFD_ERR_ARG without a free surface. */
#define CGFD_NPEAK 15
int cgfd_get_surface_peaks(cgfd_solver *s, float *out);

/* One wavefield component (CGFD_VX..CGFD_TXY) of the current level at
 * interior points, [nk][nj][ni]. */
int cgfd_get_wavefield(cgfd_solver *s, int cmp, float *out);

/* Overwrite one component of the current level at interior points (ghosts
 * stay zero), [nk][nj][ni].  For initial conditions and tests; the
 * reference always starts from rest (alloc.cu:543-551). */
int cgfd_set_wavefield(cgfd_solver *s, int cmp, const float *in);

/* Size in bytes of a checkpoint of the full solver state. */
int cgfd_checkpoint_size(cgfd_solver *s, unsigned long long *bytes);
/* Copy the full time-stepping state (wavefield, PML auxiliaries, fault
 * wavefield and fault state, step counter) to host memory `buf`. */
int cgfd_checkpoint(cgfd_solver *s, void *buf, unsigned long long bytes);
/* Restore a state written by cgfd_checkpoint on a solver created from the
 * same configuration. */
int cgfd_restore(cgfd_solver *s, const void *buf, unsigned long long bytes);

/* Kernel launches issued by the last cgfd_run call (for accounting). */
int cgfd_last_launches(const cgfd_solver *s, long long *launches);

/* 1: time every volume-stage launch with CUDA events on the solver's
 * stream (cgfd_run reads each step's events 8 steps later, so the host
 * never waits on the step in flight); 0: off (default).  Switching builds
 * the step graphs of the new mode if they do not exist yet (cgfd_upload
 * builds those of the default mode), so that no graph is captured or
 * instantiated inside a run. */
int cgfd_set_timing(cgfd_solver *s, int on);
/* Device time of the last cgfd_run (events on the solver's stream at its
 * start and end) and, with timing on, the summed duration and count of its
 * volume-stage launches. */
int cgfd_last_timing(const cgfd_solver *s, double *run_ms, double *volume_ms,
                     long long *volume_launches);
/* Per-kernel detail of the last cgfd_run with timing on (no counterpart in
 * the reference; instrumentation for roofline figures).  which = 0: the
 * volume stage (all volume kernels of one RK stage); which = 1: the
 * interior-box kernel alone.  ms: summed device time of the timed launches;
 * launches: their number; points: grid points one launch updates. */
int cgfd_last_kernel_timing(const cgfd_solver *s, int which, double *ms,
                            long long *launches, long long *points);

/* Advance nsteps time steps exactly like cgfd_run, allocating nothing
 * (no counterpart in the reference).
 *
 * For callers that cannot allocate between steps.  Examples: a loop that
 * shares the device with other work under a fixed memory budget, where
 * every byte is already claimed.  Or a time-sliced loop that interleaves
 * this solver with other GPU work and cannot afford the device-wide
 * synchronisation that cudaMalloc / cudaFree may imply.  cgfd_run does
 * allocate on first use: each of the 8 operator pairs is captured once as a
 * CUDA graph, and instantiating a graph allocates host and device memory.
 * This entry point instead launches the kernels of each step directly on
 * the solver's stream.  It calls no allocating CUDA or library routine,
 * and its error messages go to a fixed per-thread buffer.
 *
 * Scratch.  The fault kernels need one scratch buffer per RK stage (the
 * tractions around the split nodes).  Here it is a fixed device array of
 * CGFD_NOALLOC_SCRATCH_FLOATS floats (32 MiB), one per device, in the
 * library's static device memory: a GPU holds those 32 MiB from the time
 * the CUDA runtime loads this part of the library's device code on it (at
 * the latest, the first call of this entry point on that GPU; with eager
 * module loading, when the library's context starts) until the process
 * exits.  Each fault needs
 * 108 * (nj_split + 6) * (nk_split + 6) floats, where nj_split x nk_split
 * is the bounding box of its split nodes, rounded up to a multiple of 64.
 * Every fault of the solver takes its own slice of the array, because the
 * first fault kernels of a stage run for all faults before the later ones
 * run for any of them; so the SUM over the solver's faults sets the need.
 * A solver whose faults need more than the array holds is rejected with
 * CGFD_ERR_ARG before anything runs.  Nothing in the array has to start at
 * zero: every stage writes each element it reads.
 *
 * Set-up.  The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress) and keeps it for later calls on that device; the
 * address stays valid for the life of the device's primary context (a
 * cudaDeviceReset invalidates it, so do not reset a device between calls).
 * The look-up may also load the library's device code for that device.
 * Make this first call before any stream capture.  Call with the solver's
 * device current, as for every entry point.  Timing (cgfd_last_timing) is
 * not measured here and reads 0 after this call.
 *
 * Concurrency.  The array is shared by all solvers on a device.  Calls on
 * the same device must not overlap: not from two threads, and not on two
 * streams.  Overlapping calls race on the scratch and corrupt both results.
 * Calls on different devices are independent.  Mixing cgfd_run and
 * cgfd_run_noalloc on one solver is allowed; the state carries over.
 *
 * Returns like cgfd_run: CGFD_ERR_UNSTABLE on a non-finite slip rate or
 * station value, CGFD_ERR_CUDA on a launch failure. */
#define CGFD_NOALLOC_SCRATCH_FLOATS (8u * 1024u * 1024u)
int cgfd_run_noalloc(cgfd_solver *s, int nsteps);

/* Ensembles (no counterpart in the reference: the batched-scenario form of
 * the forward run).  A set of independent solvers, typically scenarios of
 * different sizes, stress fields and nucleation points, advanced together:
 * each time step of all members is one CUDA graph launch whose branches are
 * the members' steps, each on its member's own stream, so that scenarios too
 * small to fill the GPU alone run side by side.  Members stay owned by the
 * caller, must live on the current device, must have taken the same number
 * of steps, and must outlive the ensemble; read their results with the
 * usual getters.  Calling cgfd_run on a member between ensemble runs puts
 * it out of step: cgfd_ensemble_run then returns CGFD_ERR_STATE. */
typedef struct cgfd_ensemble cgfd_ensemble;
int cgfd_ensemble_create(cgfd_solver *const *members, int n, cgfd_ensemble **out);
/* Advance every member by nsteps time steps.  Returns the first member
 * error (CGFD_ERR_UNSTABLE, ...) with the member's index in the message. */
int cgfd_ensemble_run(cgfd_ensemble *e, int nsteps);
void cgfd_ensemble_destroy(cgfd_ensemble *e);

/* Release device and host memory of the handle. */
void cgfd_destroy(cgfd_solver *s);

/* Message of the last error of the calling thread ("" if none). */
const char *cgfd_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* CGFD_H */
