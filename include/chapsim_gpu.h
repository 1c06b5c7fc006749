/*
 * chapsim_gpu.h -- C ABI of the B200 (sm_100a) CHAPSim2 per-timestep hot path.
 *
 * The library owns all device state of one domain (velocity, pressure, RK3
 * history, work arrays), resident in HBM across steps.  Host arrays use the
 * reference's Fortran x-pencil layout: column-major, x fastest, full domain.
 * Every entry point returns 0 on success and a non-zero chs_status otherwise;
 * chs_last_error() returns the message.  A handle is bound to one CUDA stream
 * and must be used from one host thread at a time.
 *
 * Each entry point names the reference routine it replaces (file:line in
 * weiwangstfc/CHAPSim2).
 */
#ifndef CHAPSIM_GPU_H
#define CHAPSIM_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct chs_handle chs_handle;

enum chs_status {
  CHS_OK = 0,
  CHS_ERR_ARG = 1,       /* invalid argument or unsupported configuration */
  CHS_ERR_CUDA = 2,      /* CUDA runtime error */
  CHS_ERR_STATE = 3,     /* call not valid in the current state */
  CHS_ERR_NUMERIC = 4    /* NaN/Inf detected in the solution */
};

/* field identifiers for upload/download */
enum chs_field {
  CHS_QX = 0, CHS_QY = 1, CHS_QZ = 2, CHS_PRES = 3, CHS_PCOR = 4,
  CHS_MX_RHS0 = 5, CHS_MY_RHS0 = 6, CHS_MZ_RHS0 = 7,
  /* variable-property runs (after chs_thermo_init): fl%gx..gz, tm%rhoh, tm%hEnth, tm%tTemp,
   * tm%kCond, fl%dDens, fl%mVisc, tm%ene_rhs0 */
  CHS_GX = 8, CHS_GY = 9, CHS_GZ = 10, CHS_RHOH = 11, CHS_HENTH = 12, CHS_TTEMP = 13,
  CHS_KCOND = 14, CHS_DDENS = 15, CHS_MVISC = 16, CHS_ENE_RHS0 = 17
};

/* precision of the path */
enum chs_precision { CHS_FP64 = 0, CHS_MIXED = 1 };

/*
 * Domain configuration: the scalars of t_domain/t_flow that the momentum and
 * Poisson routines read (src/modules.f90:412-653), the nominal boundary codes
 * as read from [boundary] (src/input_general.f90:399-424) and the y geometry
 * built by Buildup_geometry_mesh_info (src/geometry.f90:410-530).
 */
typedef struct chs_config {
  int nc[3];                /* cells in x, y, z */
  int iacc;                 /* 1 CD2, 2 CD4, 3 CP4, 4 CP6 (src/modules.f90:248-251) */
  int istret;               /* 0 none, 1 centre, 2 two-sided, 3 bottom, 4 top */
  int ifft;                 /* 2 FISHPACK x/z-FFT + y-TDMA (tanh mapping), 3 3D FFT (src/modules.f90:169-170):
                             * poisson_000 for periodic y, poisson_010 for y walls
                             * (src/poisson_1stderivcomp.f90:794-820; even ny, istret 0, 1 or 2, whose
                             * y arrays below must be the 3FMD mapping, src/geometry.f90:287-408) */
  int idriven;              /* 0 none, 1 constant x mass flux */
  int precision;            /* chs_precision */
  double lxx, lyt, lyb, lzz;
  double rstret, dt, ren;
  int nominal_bc[3][5][2];  /* [x,y,z][qx,qy,qz,p,T][side] bc codes (src/modules.f90:223-229) */
  double fbcy_const[5][2];  /* constant y-wall values [qx,qy,qz,p,T][side] */
  const double* yp;         /* nc[1]+1 node coordinates */
  const double* yc;         /* nc[1] centre coordinates */
  const double* ymap_pt;    /* yMappingpt(:,1), nc[1]+1 */
  const double* ymap_cc;    /* yMappingcc(:,1), nc[1] */
} chs_config;

/*
 * Variable-property set-up: the nondimensional property table (ftplist after
 * Buildup_thermo_mapping_relations, src/input_thermo.f90:600-693), sorted by
 * increasing T with rho*h increasing, 1/(Re Pr) (Update_PrGr,
 * src/tools_solver.f90:49-87) and the initial uniform temperature.
 */
typedef struct chs_thermo {
  int ntable;
  const double *t, *h, *d, *m, *k, *cp, *b;  /* T, h, rho, mu, kappa, cp, beta columns */
  double rPrRen;
  double t_ini;
} chs_thermo;

typedef struct chs_diag {
  double max_div;      /* max |div u| over the domain (Check_element_mass_conservation, src/eq_continuity.f90:337-397) */
  double bulk_ke;      /* bulk kinetic energy (write_monitor_total, src/io_monitor.f90:209-241) */
  double bulk_u;       /* volume-averaged qx */
  double last_bulk_rhs;/* last mass-flux correction removed from mx_rhs */
  int nan_flag;        /* 1 if a NaN/Inf was found */
  double mcon[3];      /* Check_element_mass_conservation's monitors (src/eq_continuity.f90:379-389): max |div|
                          over the x slabs i = 1:4, 5:n-4 and n-5:n (1-based), the fl%mcon(1:3) of the reference */
} chs_diag;

/* Replaces initialise_fft / Prepare_LHS_coeffs_for_operations / allocation
 * (src/chapsim.f90:79-97, src/poisson_interface.f90:102-116,
 * src/basics_operations2.f90:1600-1800).  device < 0 uses the current device. */
int chs_create(const chs_config* cfg, int device, chs_handle** out);
int chs_destroy(chs_handle* h);

/* Copy one field between host (Fortran layout) and the handle's device state.
 * n is the element count and must equal the field's staggered size. */
int chs_upload_field(chs_handle* h, int field, const double* host, size_t n);
int chs_download_field(chs_handle* h, int field, double* host, size_t n);

/* Replaces Solve_momentum_eq(fl, dm, isub) (src/eq_momentum2.f90:1799-1932):
 * momentum RHS, RK3 fractional step, mass-flux driving, Poisson solve,
 * pressure update, projection.  isub = 0 is the initial Euler step
 * (src/chapsim.f90:135), isub = 1..3 the RK3 substeps. */
int chs_momentum_substep(chs_handle* h, int isub);

/* nsteps full RK3 steps (3 substeps each) of the time loop
 * (src/chapsim.f90:243-309), replayed from a captured CUDA graph. */
int chs_step(chs_handle* h, int nsteps);

/* Replaces solve_fft_poisson(rhs_xpencil, dm) (src/poisson_interface.f90:119-149)
 * on a host buffer of nc[0]*nc[1]*nc[2] values, in place. */
int chs_poisson_solve(chs_handle* h, double* rhs_inout);

/* Drop-in for Solve_momentum_eq with host-owned arrays (the Fortran x-pencil
 * arrays fl%qx, fl%qy, fl%qz, fl%pres): uploads them, runs the substep and
 * copies the updated fields back (in place).  Pinned host memory
 * (chs_host_alloc) makes the copies asynchronous DMA. */
int chs_momentum_substep_host(chs_handle* h, int isub, double* qx, double* qy, double* qz, double* pres);

/* Time nsteps RK3 steps replayed from the captured graphs with CUDA events
 * recorded on the handle's stream; *ms = elapsed device time. */
int chs_time_steps(chs_handle* h, int nsteps, float* ms);

/* Time nsteps RK3 steps of chs_momentum_substep_host (host->device copies,
 * substep, device->host copies, three times per step) with CUDA events on the
 * handle's stream; *ms = elapsed device time including the copies. */
int chs_time_steps_host(chs_handle* h, int nsteps, double* qx, double* qy, double* qz, double* pres, float* ms);

/* Like chs_time_steps_host for any set of fields (chs_field ids): every substep
 * copies the listed host arrays in, replays the substep graph (energy and
 * momentum for variable-property runs) and copies them back.  This is the
 * host-array drop-in of one time-loop substep (src/chapsim.f90:292-309) for a
 * caller that keeps those arrays on the host.  The copies run on two internal
 * streams, one per direction, ordered per field (a field's copy-in for the
 * next substep follows its copy-out), so the host arrays must be page-locked
 * (chs_host_alloc) for the directions to overlap and must not be touched by
 * the caller until the call returns; all work is complete on return. */
int chs_time_steps_host_fields(chs_handle* h, int nsteps, int nfields, const int* ids, double* const* bufs,
                               float* ms);

/* The same with the host arrays copied in at the start and out at the end of
 * every RK3 step (src/chapsim.f90:243-391, one pass of the time loop): the
 * caller that owns the state on the host between time steps.  A field's
 * copy-in for the next step follows its copy-out, and with variable
 * properties the energy part of the first substep starts once its fields are
 * in.  Same buffer rules as chs_time_steps_host_fields. */
int chs_time_rk3_host_fields(chs_handle* h, int nsteps, int nfields, const int* ids, double* const* bufs,
                             float* ms);

/* Page-locked host buffers for the host-array entry points. */
void* chs_host_alloc(size_t bytes);
void chs_host_free(void* p);

/* Per-kernel profile of one substep (not graph-replayed): for each launch, its
 * class (0 line op, 1 FFT, 2 y solve, 3 elementwise/reduction, 4 fused CD2
 * kernel: a momentum component or the energy equation), direction
 * (-1 if none), algorithmic bytes moved and CUDA-event duration. */
typedef struct chs_kprof {
  int kind;
  int dir;
  double bytes;
  float ms;
} chs_kprof;
int chs_profile_substep(chs_handle* h, int isub, chs_kprof* out, int max, int* n);
/* The same profile taken inside a CUDA graph of the substep (isub 1..3): the
 * substep is captured on one stream with an event-record node around every
 * launch and replayed once, so each duration is the launch's time in graph
 * replay (the timed path) rather than after an eager launch.  Advances the
 * state by that substep, like chs_momentum_substep. */
int chs_profile_substep_graph(chs_handle* h, int isub, chs_kprof* out, int max, int* n);
/* In-step time of one kernel class: the substep isub (1..3) is captured as the
 * timed path captures it (dataflow lanes included) with only the launches of
 * class `kind` (0 line op, 1 FFT, 2 y solve, 3 elementwise/reduction, 4 fused
 * CD2 kernels; -1 all of them), the graph is replayed reps times after one
 * warm-up, and *ms is the mean time of one replay: the class's time without
 * the per-launch event nodes of chs_profile_substep_graph.  The state is saved
 * before and restored after (device memory for one copy of the handle's fields
 * is allocated for the duration of the call).  No counterpart in the reference. */
int chs_profile_class(chs_handle* h, int isub, int kind, int reps, float* ms);

/* Replaces Buildup_thermo_mapping_relations + initialise_thermal_properties
 * (src/chapsim.f90:103-108, src/input_thermo.f90:1070-1103) and the q -> g
 * conversion of the initial field (src/initialisation.f90:389).  Call once,
 * after the velocity has been uploaded.  Needs the channel (y walls at rest,
 * Neumann T there, x and z periodic); the wall dT/dy values are the config's
 * fbcy_const[4][side]. */
int chs_thermo_init(chs_handle* h, const chs_thermo* th);

/* Replaces Solve_energy_eq(fl, tm, dm, isub) (src/eq_energy.f90:405-458):
 * energy RHS, RK3 fractional step, rho*h update and the property update of
 * Update_thermal_properties (src/eq_energy.f90:14-146).  isub 1..3.  In a
 * variable-property run chs_momentum_substep then advances g and converts it to
 * q, and chs_step runs both equations per substep. */
int chs_energy_substep(chs_handle* h, int isub);

/*
 * MLP surrogate of the per-cell property update of Update_thermal_properties
 * (src/eq_energy.f90:14-146): a 1 -> 64 -> 64 -> 64 -> 4 tanh network from rho*h
 * to (T, rho, mu, kappa), trained on the GPU by this library's own FP32
 * forward/backward/Adam kernels on seeded samples whose targets are the table
 * lookup, evaluated with BF16 tensor cores (FP32 accumulation).  In mode 1 the
 * network's T of each cell gives the table row where the rho*h search starts;
 * the table judges it exactly (a start within tol of the T range that brackets
 * the cell's rho*h is verified, else the search runs from scratch: the
 * fallback), so the stored properties equal the table lookup's bit for bit.
 * No counterpart in the reference.
 */
typedef struct chs_mlp_train_cfg {
  int nsamples;                /* training samples (e.g. 1000000) */
  int batch;                   /* minibatch size */
  int epochs;
  double lr;                   /* Adam learning rate (cosine decay to 1%) */
  unsigned long long seed;
} chs_mlp_train_cfg;

typedef struct chs_mlp_report {
  double final_loss;           /* last minibatch mean squared error (normalised outputs) */
  double train_ms;             /* device time of the training loop */
  int steps;
} chs_mlp_report;

int chs_mlp_train(chs_handle* h, const chs_mlp_train_cfg* cfg, chs_mlp_report* rep);
/* mode 0: table lookups (the reference's method); 1: the network's T picks the table row where the
 * rho*h search starts, within tol (> 0 sets it) of the table's T range; the table verifies that
 * start and otherwise searches from scratch (fallback), so the properties are always exactly the
 * table lookup's */
int chs_mlp_set_mode(chs_handle* h, int mode, double tol);
/* cells that took the table fallback since the last chs_mlp_set_mode */
int chs_mlp_fallbacks(chs_handle* h, unsigned long long* count);
/* get (set = 0) or set (set = 1) the flat FP32 parameters (n = 8708) */
int chs_mlp_params(chs_handle* h, float* buf, int n, int set);
/* loss and gradients of the FP32 network for B samples (normalised x[B], targets t[B][4]) */
int chs_mlp_grad(chs_handle* h, const float* params, int B, const float* x, const float* t, float* grad,
                 float* loss);
/* tensor-core inference on n host values of rho*h: out[5][n] = T, rho, mu, kappa, h.  tol < 0: the
 * network's own outputs (no table); tol = 0: the table search alone; tol > 0: as
 * chs_mlp_set_mode; *nfallback = cells whose network start row was not verified */
int chs_mlp_eval(chs_handle* h, int n, const double* rhoh, double tol, double* out, unsigned long long* nfallback);
/* normalisation: out[10] = xa, xb (x = xa*rhoh + xb), ya[4], yb[4] (value = ya*y + yb) */
int chs_mlp_norm(const chs_handle* h, double* out);

/*
 * Batched ensembles (no counterpart in the reference, which runs one domain per
 * MPI job): independent handles, of any grids, Reynolds numbers and precisions,
 * on one device advance together.  Each RK3 substep is one captured CUDA graph
 * whose branches are the members' substeps on their own streams, so one graph
 * launch advances every member and the members' kernels overlap on the GPU.
 * The members stay owned by the caller and must have taken their initial step
 * (chs_momentum_substep(h, 0)); their own entry points stay usable and are
 * ordered after the ensemble's work.
 */
typedef struct chs_ensemble chs_ensemble;
int chs_ensemble_create(chs_handle* const* members, int n, chs_ensemble** out);
int chs_ensemble_step(chs_ensemble* e, int nsteps);
int chs_ensemble_time_steps(chs_ensemble* e, int nsteps, float* ms);
long long chs_ensemble_kernel_launches(const chs_ensemble* e);
int chs_ensemble_destroy(chs_ensemble* e);

/* Autotuner: times nsteps RK3 steps for each candidate launch shape (explicit
 * line operators: the specialised kernels, block 0, or the generic kernel with
 * a CTA size of 128/256/512; lines per CTA of the compact-scheme tile;
 * separate operators or fused per-component sums) on this handle, restoring
 * the state after each trial, and keeps the fastest. */
int chs_autotune(chs_handle* h, int nsteps, int* block, int* lt_max, int* fused, float* best_ms);
/* Set the launch shape directly (e.g. the one chs_autotune found for another
 * handle of the same grid): block 0/128/256/512, lt_max 0/16/32/64, fused 0/1;
 * 0 selects the defaults. */
int chs_set_launch_shape(chs_handle* h, int block, int lt_max, int fused);
/* Streams a captured substep graph spreads its launches over (1..8; default 3
 * for CHS_FP64, 4 for CHS_MIXED).
 * Each launch waits only for the launches whose buffers it reads or overwrites,
 * so independent operators run concurrently; 1 keeps program order on one
 * stream.  Results are identical for every setting (no counterpart in the
 * reference, which runs the operators one after another). */
int chs_set_lanes(chs_handle* h, int lanes);
/* Fused substep kernels for the CD2 scheme: on = 1 (the default) forms the
 * momentum right-hand sides of all three components with the fractional step
 * in one pass that evaluates every interpolation and derivative where it is
 * needed (the same plans, boundary rows and arithmetic as the operator path
 * of Compute_momentum_rhs, src/eq_momentum2.f90:101-1571, without writing
 * them to device memory), likewise the energy right-hand side and the
 * projection; on = 0 runs one operator per derived quantity.  The other
 * schemes (CD4, CP4, CP6) always take the operator path.  No counterpart in
 * the reference, which has only the operator path. */
int chs_set_fusion(chs_handle* h, int on);

/*
 * Restart files and running statistics.  Files follow the reference's naming
 * (generate_pathfile_name, src/io_tools.f90:44-61): <dir>/domain<idom>_<keyword>_<iter>.bin,
 * each the raw FP64 full-domain array in Fortran order as decomp_2d_write_one writes it on one
 * rank (no header).
 *
 * chs_write_restart: qx, qy, qz, pr (+ rhoh, temp with variable properties) -- replaces
 *   write_instantanous_flow / _thermo (src/io_restart.f90:71-108).
 * chs_read_restart: reads them, pcor = 0, and with variable properties the property update from
 *   rho*h (wall states included) and g = q * rho_face -- replaces read_instantanous_flow /
 *   _thermo and restore_*_variables_from_restart (src/io_restart.f90:112-226).  The next
 *   substep 1 continues the run (its RK3 history weight is zero).
 * chs_stats_update: running means of p, u_i (cell-centre P2C interpolations) and u_i u_j (+ T,
 *   T^2), sample nstat = iteration - stat_istart + 1 -- replaces update_statistics_flow /
 *   _thermo (src/post_statistics.f90:152-283); FP64 accumulation in every precision.
 * chs_stats_get: which 0 pr, 1-3 ux uy uz, 4-9 uu vv ww uv uw vw, 10 T, 11 TT (n = nc1*nc2*nc3).
 * chs_write_statistics / chs_read_statistics: the time_averaged_* files of
 *   write_statistics_flow / _thermo and read_statistics_* (src/post_statistics.f90:98-148,
 *   217-239, 285-296).
 * chs_data_file_name: the file name for a keyword (host only).
 */
int chs_write_restart(chs_handle* h, const char* dir, int idom, int iter);
int chs_read_restart(chs_handle* h, const char* dir, int idom, int iter);
int chs_stats_update(chs_handle* h, int nstat);
int chs_stats_get(chs_handle* h, int which, double* host, size_t n);
int chs_write_statistics(chs_handle* h, const char* dir, int idom, int iter);
int chs_read_statistics(chs_handle* h, const char* dir, int idom, int iter);
int chs_data_file_name(const char* dir, int idom, const char* keyword, int iter, char* buf, size_t len);

/* Same as chs_poisson_solve on a device buffer (no host copies). */
int chs_poisson_solve_device(chs_handle* h, double* d_rhs_inout);

/* Post-step checks (src/chapsim.f90:326-356): divergence, bulk KE, NaN scan. */
int chs_diagnostics(chs_handle* h, chs_diag* out);

/* One compact operator Get_{x,y,z}_{midp,1der}_{C2P,P2C,C2C,P2P}_3D
 * (src/basics_operations2.f90:3952-4800) on host arrays.
 * dir 0/1/2; fam 0 d1C2C, 1 d1P2P, 2 d1C2P, 3 d1P2C, 4 m1C2P, 5 m1P2C;
 * nin3 = input extents (x,y,z); fbc2d, when non-NULL, holds the 4 boundary
 * planes in the reference layout fbcx(4,n2,n3) / fbcy(n1,4,n3) / fbcz(n1,n2,4). */
int chs_op3d(chs_handle* h, int dir, int fam, int ibc1, int ibc2, const double* fbc2d,
             const double* in, const int nin3[3], double* out);

/* Host-only inspection of the operator plan that chs_op3d / the substep would use
 * (test support; no counterpart in the reference, no device work).  Writes the
 * bulk stencil, boundary rows, pre-factorised LHS and y metric into buf
 * (len >= 128 + 5*nout doubles); see chs_solver.cu for the layout. */
int chs_plan_inspect(const chs_config* cfg, int dir, int fam, int ibc1, int ibc2, int has_fbc, double* buf,
                     size_t len);

/* Block until all work queued on the handle's stream is done. */
int chs_sync(chs_handle* h);

/* Number of kernels the handle launched since creation (all entry points). */
long long chs_kernel_launches(const chs_handle* h);

/* Last error message (NUL-terminated, truncated to len). */
int chs_last_error(const chs_handle* h, char* buf, size_t len);

/* Periodic 3D pressure Poisson solve that allocates nothing.  No counterpart in
 * the reference (it is the spectral solve of poisson_000,
 * src/poisson_1stderivcomp.f90:1016-1195, without a handle).
 *
 * For callers that cannot allocate device memory (a host code whose device
 * memory is owned by its own pool, or a fixed-footprint deployment): solves
 * L phi = rhs in place on the caller's device array d_rhs (nc[0]*nc[1]*nc[2]
 * doubles, x fastest) for a box of edge lengths len[3], periodic in x, y and z,
 * with the modified wavenumbers of the C2P derivative of scheme iacc (1 CD2,
 * 2 CD4, 3 CP4, 4 CP6).  The result equals chs_poisson_solve_device on a handle
 * of the same grid and scheme.  Kernels run on `stream` (a cudaStream_t; NULL
 * is the legacy default stream).
 *
 * Work memory is a fixed module-level device array of 16 MiB + 288 KiB (spectrum
 * 16 MiB, twiddles 192 KiB, squared wavenumbers 96 KiB), so the
 * limits are (nc[0]/2+1)*nc[1]*nc[2] <= 1048576 complex values and each nc[d]
 * <= 4096, each of the form 2^a 3^b; larger grids return CHS_ERR_ARG with a
 * message.  Nothing in it needs to start at zero: every value is written before
 * it is read.  The first call on a device, and any call whose nc, len or iacc
 * differ from the previous call's, does set-up: it writes the FFT and
 * wavenumber tables with a host-to-device copy on `stream` and synchronizes
 * that stream, so make such a call before any stream capture.  The tables are
 * tied to the device context: after cudaDeviceReset the next call sets up
 * again.  A set-up holds a per-device lock only.  All calls on one
 * device share the one work array: calls that overlap in time (on different
 * streams, or from threads that do not order them) race and corrupt each other;
 * order them on one stream.  Errors are written to err (errlen bytes, may be
 * NULL) and returned as chs_status. */
int chs_poisson_periodic_static(double* d_rhs, const int nc[3], const double len[3], int iacc, void* stream,
                                char* err, size_t errlen);

#ifdef __cplusplus
}
#endif

#endif /* CHAPSIM_GPU_H */
