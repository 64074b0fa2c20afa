/*
 * lare_gpu.h - C ABI of the B200 (sm_100a) Lagrangian-remap timestep.
 *
 * The reference (Warwick-Plasma/Lare3d, Fortran 90) advances its state with
 * argument-less module procedures that operate on the `shared_data` globals:
 *
 *   src/core/lare3d.f90:84   CALL lagrangian_step        (lagran.F90:50)
 *   src/core/lare3d.f90:85   CALL eulerian_remap(step)   (remap.f90:33)
 *   src/core/lare3d.f90:87   CALL eta_calc               (lagran.F90:1176)
 *   src/core/lare3d.f90:88   CALL output_routines(step)  (diagnostics.F90:43,
 *                            of which energy_account :517 is the hot part)
 *
 * This library owns a device-resident copy of that state and replaces those
 * calls one for one.  Every array argument is a Fortran column-major array
 * with exactly the ghost-inclusive bounds the reference allocates
 * (mpi_routines.F90:295-327):
 *
 *   cell  rho, energy, eta         (-1:nx+2, -1:ny+2, -1:nz+2)
 *   node  vx, vy, vz, visc3        (-2:nx+2, -2:ny+2, -2:nz+2)
 *   face  bx                       (-2:nx+2, -1:ny+2, -1:nz+2)
 *         by                       (-1:nx+2, -2:ny+2, -1:nz+2)
 *         bz                       (-1:nx+2, -1:ny+2, -2:nz+2)
 *   1-D   dxb (-1:nx+2), dxc (-1:nx+1), likewise y and z; grav (-1:nz+2)
 *
 * so that a Fortran driver passes its own arrays through iso_c_binding with
 * no repacking.  All entry points return 0 on success and a negative
 * LARE_E* code on failure; lare_gpu_last_error() gives the message.  A
 * context is not thread-safe; it owns one CUDA stream.
 */
#ifndef LARE_GPU_H
#define LARE_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

/*
 * Boundary codes, shared_data.F90:65-66.  A direction is periodic only when
 * both its sides are (else LARE_EINVAL at init).  BC_OPEN sides get the
 * characteristic boundaries of openboundary.f90 once per step; their second
 * ghost layer (as uploaded) is the far field and is never overwritten.
 */
#define LARE_BC_PERIODIC 1
#define LARE_BC_USER 2
#define LARE_BC_OPEN 3

/* Status codes. */
#define LARE_OK 0
#define LARE_EINVAL (-1)     /* bad argument, size or unsupported option */
#define LARE_ECUDA (-2)      /* CUDA runtime error */
#define LARE_ENOMEM (-3)     /* device allocation failed */
#define LARE_EDT (-4)        /* dt underflow / non-finite dt from set_dt */
#define LARE_ESTAGES (-5)    /* RKL2 stage count not representable */
#define LARE_ENOTFOUND (-6)  /* unknown field name */
#define LARE_ENONFINITE (-7) /* non-finite value in uploaded state */
#define LARE_ETOOLARGE (-8)  /* grid beyond 32-bit indexing or a fixed-capacity entry point's limit */
#define LARE_EEOS (-9)       /* neutral_fraction's temperature bracket is empty (neutral.f90:171-174) */

/* Precision codes of lare_gpu_init. */
#define LARE_FP64 64        /* FP64 drop-in: FMA contraction, shared reciprocals */
#define LARE_FP64_EXACT 65  /* FP64, the reference's arithmetic bit for bit */
#define LARE_FP32 32        /* FP32 form */

/* Equations of state, shared_data.F90:73 (0 is taken as EOS_IDEAL). */
#define LARE_EOS_IDEAL 1
#define LARE_EOS_ION 2
#define LARE_EOS_PI 3

/*
 * Control scalars read by the hot path.  Field names follow
 * src/control.f90 and src/core/shared_data.F90.
 */
typedef struct lare_params {
  double gamma;            /* ratio of specific heats (setup.F90:46, control.f90:42) */
  double visc1, visc2;     /* shock viscosity coefficients (control.f90:85-86) */
  double eta_background;   /* background resistivity (control.f90:119) */
  double eta0, j_max;      /* anomalous resistivity and current threshold (:121-126) */
  double kappa_0;          /* normalised Spitzer conductivity (normalise.f90:54-55) */
  double flux_limiter;     /* Larsen flux limiter (control.f90:134) */
  double ionise_pot;       /* normalised ionisation potential, 0 unless EOS_ION (normalise.f90:48) */
  double xi_n;             /* neutral fraction, a constant 0 or 1 under EOS_IDEAL (lare3d.f90:72) */
  double va_max;           /* Boris Alfven speed limit (control.f90:184) */
  double dt_multiplier;    /* CFL safety factor, 0.9 in the reference (shared_data.F90:60) */
  double dt_from_restart;  /* dt used by the first set_dt after a restart (lagran.F90:1080-1086) */
  double kappa_perp_ratio; /* extension: kappa_perp / kappa_par; 0 reproduces the reference */
  int resistive_mhd;       /* control.f90:117 */
  int conduction;          /* control.f90:130 */
  int heat_flux_limiter;   /* control.f90:132 */
  int use_viscous_damping; /* control.f90:89 */
  int boris;               /* control.f90:183 */
  int restart;             /* IC_RESTART (lare3d.f90:56-60) */
  int xbc_min, xbc_max, ybc_min, ybc_max, zbc_min, zbc_max; /* control.f90:169-174 */
  /*
   * Partially ionised plasma (neutral.f90).  With eos_number EOS_ION or
   * EOS_PI the neutral fraction xi_n becomes a per-cell array that
   * neutral_fraction solves for; with cowling_resistivity the cross-field
   * resistivity eta_perp (perpendicular_resistivity) enters set_dt and the
   * resistive fluxes.  The constants are the normalised values the
   * reference holds after setup_neutral (neutral.f90:31-63) and
   * normalise_transport (normalise.f90:39-51); xi_n above is then unused.
   */
  int eos_number;          /* LARE_EOS_* (control.f90:191) */
  int cowling_resistivity; /* control.f90:162 */
  double f_bar, t_bar, r_bar, tr, eta_bar;
  /*
   * Optically thin radiative losses (radiative.f90:98-208, lagran.F90:174-
   * 178): Townsend's exact integration of the reference's default piecewise
   * power-law loss function.  temp_norm and time_norm are normalise.f90's
   * (:32-34); rho_norm and mf are control.f90's (:46, :60).
   */
  int radiation;
  double temp_norm, time_norm, rho_norm, mf;
  /*
   * rke (control.f90): the momentum remap records the kinetic energy it
   * loses per cell ([xyz]remap.f90, x_momx_flux :664-695 and siblings) and
   * energy_correction returns it to the internal energy after the remap.
   */
  int rke;
  /*
   * cooling_term (control.f90:205-206): exponential moving averages, weight
   * alpha_av, of the viscous heating (lagran.F90:464-475) and of the ohmic
   * heating (:1290-1302) are taken off the energy each step; the averages
   * persist across steps (fields "cool_term_v", "cool_term_b").
   */
  int cooling_term;
  double alpha_av;
  /*
   * coronal_heating (control.f90:142): each step, after the pressure is
   * formed and before the shock viscosity (lagran.F90:127), the energy gains
   * heat_in * dt / rho over the whole cell array, with the dt of the previous
   * set_dt, then energy_bcs (radiative.f90:69-93 user_defined_heating).  The
   * heating rate is the user hook's: set the cell field "heat_in" (Lare
   * units, (-1:nx+2, -1:ny+2, -1:nz+2)) with lare_gpu_set_field; it is zero
   * until set and is kept between steps.
   */
  int coronal_heating;
} lare_params;

/* Scalars of shared_data that the step updates. */
typedef struct lare_scalars {
  double time, dt, dtr;                /* shared_data.F90:126 */
  double total_visc_heating;           /* shared_data.F90:133 */
  double total_ohmic_heating;
  int n_s_stages;                      /* last RKL2 stage count (conduct.f90:139) */
  int peak_substeps;                   /* lagran.F90:141 */
  int last_substeps;                   /* resistive sub-cycles of the last step */
  int steps_taken;                     /* lagrangian steps since init */
} lare_scalars;

typedef struct lare_ctx lare_ctx;

/*
 * Create a context for an nx*ny*nz grid (each >= 4).  dxb/dxc etc. are the
 * Fortran grid metrics written by setup.F90:grid (:92-247); cv is formed on
 * the device as dxb*dyb*dzb exactly as setup.F90:239-245.  precision is
 *   LARE_FP64 (64)        the FP64 drop-in: FP64 throughout, FMA contraction
 *                         and reciprocals shared between quotients, so the
 *                         last bits differ from the reference's (relative L2
 *                         within 1e-10 per field after 100 steps);
 *   LARE_FP64_EXACT (65)  FP64 with the reference's arithmetic: every multiply
 *                         and add rounded separately, IEEE quotients in the
 *                         reference's expression order, so the state equals a
 *                         gfortran x86-64 build of the reference bit for bit
 *                         (conduction's pow excepted); slower;
 *   LARE_FP32 (32)        the FP32 form: field arithmetic in FP32, dt
 *                         reduction, budgets and RKL2 coefficients in FP64.
 * Device indices are 32-bit: the padded box of an array, (nx + 5 rounded up
 * to a multiple of 4) * (ny + 5) * (nz + 5) points, must stay below 2^31,
 * else LARE_ETOOLARGE before the device is touched (a cube up to 1284^3;
 * such a grid needs about 50 arrays of 8 or 4 bytes a point, far beyond
 * one GPU's memory, which returns LARE_ENOMEM first).
 * Replaces mpi_initialise's allocation (mpi_routines.F90:295-334) for the
 * device copy.
 */
int lare_gpu_init(const lare_params* params, int nx, int ny, int nz,
                  const double* dxb, const double* dxc,
                  const double* dyb, const double* dyc,
                  const double* dzb, const double* dzc,
                  int precision, lare_ctx** out);

/* Upload the state (host Fortran arrays, bounds as in the file header). */
int lare_gpu_upload(lare_ctx* ctx, const double* rho, const double* energy,
                    const double* vx, const double* vy, const double* vz,
                    const double* bx, const double* by, const double* bz);

/*
 * Upload auxiliary arrays; any pointer may be NULL to keep the current
 * contents.  eta: cell (as left by eta_calc, lare3d.f90:68); visc3: node;
 * grav: 1-D (-1:nz+2); gamma_boris: cell (initialised to 1 by init).
 */
int lare_gpu_upload_aux(lare_ctx* ctx, const double* eta, const double* visc3,
                        const double* grav, const double* gamma_boris);

/* Set the simulation clock (time, dt) as held in shared_data. */
int lare_gpu_set_time(lare_ctx* ctx, double time, double dt);

/*
 * lagran.F90:50 lagrangian_step, including the energy/density/velocity bcs.
 * step is the driver's step counter (shared_data `step`), which the
 * predictor's half-step remap passes to eulerian_remap (lagran.F90:1057).
 */
int lare_gpu_lagrangian_step(lare_ctx* ctx, int step);

/* remap.f90:33 eulerian_remap(step): Strang-permuted x/y/z remap + bfield_bcs. */
int lare_gpu_eulerian_remap(lare_ctx* ctx, int step);

/*
 * diagnostics.F90:613 energy_correction: delta_ke (recorded by the last
 * eulerian_remap) into the energy of cells 1:n, then energy_bcs.
 * LARE_EINVAL unless rke.  lare_gpu_step and lare_gpu_run call it after the
 * remap (lare3d.f90:86).
 */
int lare_gpu_energy_correction(lare_ctx* ctx);

/* lagran.F90:1176 eta_calc. */
int lare_gpu_eta_calc(lare_ctx* ctx);

/* boundary.f90:48 boundary_conditions (b, energy, density, velocity). */
int lare_gpu_boundary_conditions(lare_ctx* ctx);

/*
 * neutral.f90:158 neutral_fraction: xi_n over the whole cell array from rho
 * and energy by bisection on the temperature (a no-op under EOS_IDEAL).
 * LARE_EEOS where a cell's temperature bracket is empty (the reference
 * stops there); the context then keeps returning LARE_EEOS from the calls
 * that check for it, like the run it replaces, so start a new context to
 * continue.  lare_gpu_step and lare_gpu_run call it first in each step
 * (lare3d.f90:83), and the resistive sub-cycles and the RKL2 stages call it
 * where the reference does (lagran.F90:147, conduct.f90:404).
 */
int lare_gpu_neutral_fraction(lare_ctx* ctx);

/*
 * neutral.f90:68 perpendicular_resistivity: eta_perp at the vertices 0:n
 * (LARE_EINVAL unless cowling_resistivity).  The resistive sub-cycles call
 * it after neutral_fraction (lagran.F90:148); a driver calls both once
 * after the initial boundary_conditions and eta_calc (lare3d.f90:70-74).
 */
int lare_gpu_perpendicular_resistivity(lare_ctx* ctx);

/*
 * One timestep of the driver loop (lare3d.f90:83-87): neutral_fraction
 * (unless EOS_IDEAL), lagrangian_step, eulerian_remap(step),
 * energy_correction (with rke), eta_calc.  time/dt (may be NULL) receive the
 * updated clock.
 */
int lare_gpu_step(lare_ctx* ctx, int step, double* time, double* dt);

/*
 * Run the driver loop from step first_step+1 until nsteps steps were taken
 * or time >= t_end (lare3d.f90:80-89).  steps_done/time/dt may be NULL.
 */
int lare_gpu_run(lare_ctx* ctx, int first_step, int nsteps, double t_end,
                 int* steps_done, double* time, double* dt);

/*
 * conduct.f90:39 conduct_heat on the current state with the given dt
 * (RKL2 super-time-stepping, stages from calc_s_stages).  Used to time the
 * conduction operator alone; n_stages (may be NULL) receives s.
 */
int lare_gpu_conduct_heat(lare_ctx* ctx, double dt, int* n_stages);

/*
 * The same RKL2 step with the stage count s given (s >= 2) instead of taken
 * from calc_s_stages.  No counterpart in the reference: it lets a
 * sub-domain copy of a grid repeat a step of the whole grid exactly (the
 * learned-conduction re-check runs plain RKL2 on windows this way).
 */
int lare_gpu_conduct_heat_stages(lare_ctx* ctx, double dt, int n_stages);

/*
 * conduct.f90:56-143 calc_s_stages alone: the RKL2 stage count s that
 * lare_gpu_conduct_heat would use for dt on the current state (it also
 * refreshes the temperature and larsen_factor arrays).  No counterpart as a
 * separate call in the reference.
 */
int lare_gpu_conduction_stages(lare_ctx* ctx, double dt, int* n_stages);

/*
 * diagnostics.F90:517 energy_account: out[0..4] = en_b, en_ke, en_int,
 * total_visc_heating, total_ohmic_heating (the en.dat record, :79-83), FP64.
 */
int lare_gpu_energy(lare_ctx* ctx, double out[5]);

/*
 * Allocation-free energy budget.  This entry point has no counterpart in the
 * reference; it computes what lare_gpu_energy returns in out[0..2] (en_b,
 * en_ke, en_int, diagnostics.F90:517-609) from the CALLER's device arrays,
 * without a context and without allocating any device memory.  It is meant
 * for callers that hold the state in their own device memory and cannot let
 * a library call cudaMalloc: a driver that owns a fixed device-memory pool,
 * or one that must not add allocations (and the device synchronisation they
 * imply) between its stream-ordered steps.
 *
 * All pointers are device pointers to the reference's Fortran-bounded
 * arrays (cell rho/energy, node vx/vy/vz, face bx/by/bz, 1-D dxb(-1:nx+2),
 * dyb, dzb); out3 is a device pointer receiving the three FP64 sums.  The
 * work is enqueued on `stream` (a cudaStream_t, NULL = default stream) and
 * the call returns without synchronising.
 *
 * Limit: (nx+1)*(ny+1)*(nz+1) <= LARE_NOALLOC_MAX_POINTS (grids up to
 * 321^3); larger grids return LARE_ETOOLARGE before any work is enqueued.
 * Its scratch is one fixed 96 KiB array in the library image that every GPU
 * loading the library keeps until the process exits.  All calls share it:
 * calls that overlap on the GPU (different streams without ordering) race
 * and give wrong sums; calls on one stream are safe.  The first call in each
 * CUDA context (per device, and again after cudaDeviceReset) looks up the
 * scratch address in that context; make that first call before any stream
 * capture begins.
 */
#define LARE_NOALLOC_MAX_POINTS 33554432
int lare_gpu_energy_noalloc(int nx, int ny, int nz, const double* rho, const double* energy,
                            const double* vx, const double* vy, const double* vz,
                            const double* bx, const double* by, const double* bz,
                            const double* dxb, const double* dyb, const double* dzb,
                            double* out3, void* stream);

/* Download the state into host Fortran arrays (any pointer may be NULL). */
int lare_gpu_download(lare_ctx* ctx, double* rho, double* energy,
                      double* vx, double* vy, double* vz,
                      double* bx, double* by, double* bz);

/*
 * Copy any named device array (the reference's variable names: "rho",
 * "vx1", "p_visc", "visc_heat", "alpha1", "cv1", "temperature", ...) to or
 * from a host buffer laid out with that array's Fortran bounds.  Used for
 * restart, SDF dumps and per-routine parity checks.
 */
int lare_gpu_get_field(lare_ctx* ctx, const char* name, double* host);
int lare_gpu_set_field(lare_ctx* ctx, const char* name, const double* host);

/* Bounds of a named array: lo[3], hi[3] (Fortran, inclusive). */
int lare_gpu_field_bounds(lare_ctx* ctx, const char* name, int lo[3], int hi[3]);

/*
 * Device address of a named array, for kernels that work on the resident
 * state in place (no counterpart in the reference).  Element (i, j, k), in
 * Fortran indices from -2 up, is origin[i + sx*j + sxy*k] (origin is the
 * address of (0, 0, 0)); elem_bytes is 8 for the FP64 engine and 4 for FP32.
 * Some arrays are double-buffered, so the address is valid only until the
 * next call that advances the state; after writing through it, call
 * lare_gpu_boundary_conditions before the next step.
 */
int lare_gpu_field_device(lare_ctx* ctx, const char* name, void** origin, int* sx, int* sxy, int* elem_bytes);

int lare_gpu_get_scalars(lare_ctx* ctx, lare_scalars* out);

/*
 * Instrumentation (not part of the reference interface).  profile(1)
 * resets and starts per-launch-site timing with CUDA events on the
 * context's stream; profile(0) stops it.  profile_report writes one line per
 * launch site, "site<TAB>launches<TAB>total ms<TAB>algorithmic bytes<TAB>
 * words per point", sorted by time, and returns the length it needs
 * (including the terminating NUL).
 */
int lare_gpu_profile(lare_ctx* ctx, int enable);
int lare_gpu_profile_report(lare_ctx* ctx, char* buf, int len);

/* Number of kernel launches issued by this context since init. */
long long lare_gpu_launch_count(lare_ctx* ctx);

/* The CUDA stream (cudaStream_t) the context launches on. */
void* lare_gpu_stream(lare_ctx* ctx);

/*
 * Block shape (bx x by threads, bx*by a multiple of 32 up to 256) of the
 * context's point kernels.  Results do not depend on it; the ensemble
 * autotuner picks it per grid size.  No counterpart in the reference.
 */
int lare_gpu_set_block(lare_ctx* ctx, int bx, int by);

const char* lare_gpu_last_error(lare_ctx* ctx);

/*
 * Self-check of the exact division the FP64 kernels use for divisions by
 * the 1-D grid metrics (a quotient corrected from the divisor's precomputed
 * reciprocal): out[i] = a[i] / b[i] computed that way, on the device
 * pointers a, b, out, enqueued on the given CUDA stream.  Every result must
 * equal the IEEE quotient bit for bit.  No counterpart in the reference.
 */
int lare_gpu_check_division(const double* a, const double* b, long long n, double* out, void* stream);

/*
 * Self-check of the reciprocal the FP64 product engine (LARE_FP64) divides
 * with: out[i] = 1 / b[i] by the hardware approximation refined by Newton-
 * Raphson steps, for b of magnitude in [2^-1000, 2^1000]; each result must be
 * within one ulp of the IEEE reciprocal.  Device pointers, enqueued on the
 * given CUDA stream.  No counterpart in the reference.
 */
int lare_gpu_check_reciprocal(const double* b, long long n, double* out, void* stream);

void lare_gpu_destroy(lare_ctx* ctx);

/*
 * Ensembles (no counterpart in the reference, which runs one simulation per
 * MPI job): n independent contexts of any sizes and parameters, advanced by
 * ONE CUDA graph launch per steps_per_launch steps of every member.  Each
 * member must have taken at least one step through lare_gpu_step (the
 * reference's first-call set-up), must not have conduction on (its RKL2
 * stage count is chosen on the host), and must not be used through other
 * calls while the ensemble exists, except after lare_ens_sync.  The
 * resistive sub-cycles run as device-side loops inside the graph.
 * steps_per_launch must be a multiple of 6 (the remap's sweep-order period,
 * remap.f90), and recorded step numbers continue from each member's count.
 *
 * lare_ens_launch enqueues nlaunch graph launches on the ensemble's stream
 * and returns; lare_ens_sync waits, folds the steps into every member's step
 * counter and returns the first LARE_E* code raised on the device (a bad dt
 * or sub-cycle count) with *first_bad its member index, or 0.
 */
typedef struct lare_ens lare_ens;
int lare_ens_create(lare_ctx* const* members, int n, int steps_per_launch, lare_ens** out);
int lare_ens_launch(lare_ens* ens, int nlaunch);
int lare_ens_sync(lare_ens* ens, int* first_bad);
void* lare_ens_stream(lare_ens* ens);
void lare_ens_destroy(lare_ens* ens);

#ifdef __cplusplus
}
#endif

#endif /* LARE_GPU_H */
