/*
 * mhit.h -- C ABI of libmhit.so, a B200 (sm_100a) implementation of one
 * MHIT36 timestep (aroccon/MHIT36).
 *
 * The reference has no plugin or operator API: its timestep is the body of
 * `do t=tstart,tfin ... enddo` in program main (multi/main.f90:329-977),
 * acting on module arrays (multi/module.f90:39-58).  These entry points
 * replace that loop body and the field set-up/I-O around it, so a Fortran
 * driver that keeps readinput, the field files and the time loop can call
 * them through iso_c_binding (see fortran/mhit_iface.f90).
 *
 * Conventions
 *   - Every call returns an int status (MHIT_OK = 0) and never exits.
 *   - A handle owns its device state and one CUDA stream; it is not
 *     thread-safe.  Distinct handles may be used concurrently.
 *   - Host arrays are Fortran order (x fastest), float64, either the
 *     reference's halo'd module shape (nx, ny+2, nz+2) or the raw interior
 *     (nx, ny, nz) of the .dat files.  The caller keeps ownership.
 */
#ifndef MHIT_H
#define MHIT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define MHIT_OK 0
#define MHIT_ERR_INVALID 1     /* bad argument (size, layout, null pointer) */
#define MHIT_ERR_CUDA 2        /* a CUDA runtime call failed */
#define MHIT_ERR_NOMEM 3       /* device allocation failed */
#define MHIT_ERR_CFL 4         /* CFL above the limit after a step (multi/main.f90:945 `stop`) */
#define MHIT_ERR_NONFINITE 5   /* NaN/Inf in the velocity reductions */
#define MHIT_ERR_IO 6          /* field file missing or of the wrong size */
#define MHIT_ERR_UNSUPPORTED 7 /* grid size or option not built */
#define MHIT_ERR_STATE 8       /* call out of order (e.g. step before set_fields) */
#define MHIT_ERR_SCRATCH_LIMIT 9 /* grid larger than the fixed scratch of mhit_poisson_noalloc */
#define MHIT_ERR_TIMEOUT 10      /* a kernel's bounded wait for staged data gave up */

/* Field layouts for set/get. */
#define MHIT_LAYOUT_RAW 0      /* (nx, ny, nz), the .dat interior (multi/readwrite.f90:29) */
#define MHIT_LAYOUT_PIX_HALO 1 /* (nx, ny+2, nz+2), the module arrays (multi/main.f90:184) */

/* Precision forms. */
#define MHIT_FP64 0            /* plain FP64 form */
#define MHIT_FP32_REFINE 1     /* FP32 state + FP64-residual Poisson refinement */

/* k^2 in the Poisson solve. */
#define MHIT_K2_SPECTRAL 0     /* -(kx^2+ky^2+kz^2), integer k: the reference (multi/main.f90:791) */
#define MHIT_K2_FD 1           /* (2/dx)^2 sum sin^2(pi m/N): exact inverse of the 7-point Laplacian */

/* Grid spacing. */
#define MHIT_GRID_REFERENCE 0  /* dx = 2pi/(nx-1) (multi/readinput.f90:37) */
#define MHIT_GRID_CONSISTENT 1 /* dx = 2pi/nx */

/*
 * input.inp lines 1-16 (multi/readinput.f90:13-31, multi/input.inp:1-16) in
 * order, then the switches of this implementation.  `lin_force` is an
 * optional 17th input.inp line (linear forcing rhs += A*u); it defaults to 0,
 * which is the reference.
 */
typedef struct mhit_params {
  int32_t restart, tstart, tfin, dump; /* lines 1-4 */
  int32_t inflow, inphi;               /* lines 5-6 */
  double dt, mu, rho;                  /* lines 7-9 */
  double f1, f2, f3, k0;               /* lines 10-13, ABC forcing */
  double radius, sigma, epsr;          /* lines 14-16 */
  double lin_force;                    /* line 17 (extension) */
  int32_t k2_mode;                     /* MHIT_K2_* */
  int32_t grid_mode;                   /* MHIT_GRID_* */
  double cfl_limit;                    /* 7.0 in the reference (multi/main.f90:945) */
  int32_t tanh_identity;               /* 1 (default): tanh(psi/(2eps)) evaluated as (2phi-1)/(1+2enum), its
                                          exact value; 0: the FP64 tanh of multi/main.f90:463-465 */
  int32_t phi_floor;                   /* 1 (default): psi from max(min(phi,1),0); 0: min(phi,1) only, as
                                          multi/main.f90:388, which makes psi NaN once phi < -1e-16 */
  int32_t reserved[6];
} mhit_params;

/* Per-step scalars (the values the reference prints or reduces). */
typedef struct mhit_diag {
  double umax;     /* gumax: signed max of u,v,w after the step (multi/main.f90:937-941) */
  double cfl;      /* gumax*dt*dxi (multi/main.f90:942) */
  double umean, vmean, wmean; /* means removed by the step (multi/main.f90:906-919) */
  double gamma;    /* ACDI gamma used by the next step (1.0*gumax, multi/main.f90:362) */
  double max_div;  /* FP32 refine form: max |div u| of the last step's FP64 projection (from 256^3 up
                      measured when mhit_step / mhit_get_diag return, from the stored ustar, p0 and
                      correction spectrum); -1 in the FP64 form */
  int64_t step;    /* steps taken since set_fields/load */
  int32_t status;  /* MHIT_OK or the sticky device error */
  int32_t reserved;
} mhit_diag;

/* FP64 diagnostics of the resident state (mhit_diagnostics). */
typedef struct mhit_stats {
  double ke;          /* 0.5 <u^2 + v^2 + w^2> over the cells */
  double dissipation; /* 2 nu <S_ij S_ij>, centred differences (post/compute_diss/main.f90:72-117) */
  double max_div;     /* max |forward-difference div u| (the projection's operator, multi/main.f90:723-725) */
  double phi_sum;     /* sum of phi over the cells (volume / dx^3) */
  double phi_min, phi_max;
  double umean;       /* mean of u after the pending mean removal */
  double reserved;
} mhit_stats;

typedef struct mhit_handle mhit_handle;

/* Fill `p` with the reference's defaults (multi/input.inp:1-16) and this
 * implementation's defaults for the extensions. */
void mhit_default_params(mhit_params* p);

/*
 * Create a simulation of nx*ny*nz cells on the current CUDA device.
 * Replaces the allocation and set-up of multi/main.f90:41-200 (MPI/cuDecomp
 * init, cuFFT plans, grid and wavenumbers, module array allocation).
 * The reference has ny = nz = nx (multi/module.f90:2-3); so does this build.
 * precision: MHIT_FP64 or MHIT_FP32_REFINE.  phase_field: 1 = ACDI on
 * (`#define phiflag 1`, multi/main.f90:39), 0 = NS only.
 */
int mhit_create(const mhit_params* p, int nx, int ny, int nz, int precision, int phase_field,
                mhit_handle** out);

/*
 * Upload the state from host arrays (copies; the caller keeps ownership)
 * and reset the time-stepping state (Euler first step, gumax = 1,
 * multi/main.f90:322-327).  phi may be NULL when phase_field = 0.
 * Replaces readfield (multi/readwrite.f90:107-207) + the halo updates of
 * multi/main.f90:249-260, 289-292.
 */
int mhit_set_fields(mhit_handle* h, const double* u, const double* v, const double* w,
                    const double* phi, int layout);

/* Download the state (any pointer may be NULL to skip that field).
 * Halo cells of MHIT_LAYOUT_PIX_HALO are filled periodically. */
int mhit_get_fields(mhit_handle* h, double* u, double* v, double* w, double* phi, int layout);

/* Download the last pressure p (multi/main.f90:842-850).  From 256^3 up the
 * FP64 step fuses the x inverse FFT into the projection and does not store
 * p; this call then recomputes it from the last step's spectrum (one x
 * inverse pass on the device) before the download.  The FP32 refinement form
 * returns p0 + dp, recomputing dp from the correction solve's spectrum the
 * same way. */
int mhit_get_pressure(mhit_handle* h, double* p, int layout);

/*
 * Advance `nsteps` timesteps: the loop body of multi/main.f90:334-946 (ACDI,
 * momentum RHS + AB2, FFT Poisson, projection, mean removal, Umax/CFL).
 * The state stays on the device; nothing is copied back except `out`
 * (may be NULL).  If a step ends with CFL > cfl_limit or a non-finite
 * reduction, the remaining steps are skipped on the device and the call
 * returns MHIT_ERR_CFL / MHIT_ERR_NONFINITE (the reference `stop`s).
 */
int mhit_step(mhit_handle* h, int nsteps, mhit_diag* out);

/*
 * FP64 diagnostics of the current state, computed on the GPU: kinetic energy,
 * viscous dissipation as the reference's post-processor computes it
 * (post/compute_diss/main.f90:72-117; pi_f32 = 1 uses its float32-rounded pi,
 * post/compute_diss/module.f90:5, with dx = 2 pi/(nx-1); pi_f32 = 0 uses the
 * grid's own dx), max |div u|, and the phi volume sum and bounds.
 */
int mhit_diagnostics(mhit_handle* h, int pi_f32, mhit_stats* out);

/*
 * Drop count and size distribution of the current phi, as the reference's
 * post-processor post/DropCountSize computes it: cells with phi >= 0.5
 * (get_interface.f90:15), 26-connected with periodic wrap (flood_fill.f90),
 * numbered in the order the x-fastest scan meets each drop's first cell
 * (get_interface.f90:28-47).  *ndrops = number of drops; for the first
 * `capacity` of them cells[i] = cell count and deq[i] = dx*(6*cells/pi)^(1/3)
 * (calculate_deq.f90:29-33), dx the handle's grid spacing.
 */
int mhit_drop_count(mhit_handle* h, int capacity, int* ndrops, int64_t* cells, double* deq);

/* Read the current per-step scalars without stepping. */
int mhit_get_diag(mhit_handle* h, mhit_diag* out);

/*
 * Write output/{u,v,w,phi}_%08d.dat under `dir` in the reference's raw
 * format (multi/readwrite.f90:1-96, called at multi/main.f90:960-971), plus
 * a sidecar `state_%08d.bin` holding rhs_o, gumax, the pending AB2 switch and
 * the step count, so that mhit_load resumes bit-exactly (the reference's
 * restart re-starts with Euler and gumax = 1, multi/main.f90:241-246, 323-325).
 */
int mhit_save(mhit_handle* h, const char* dir, int t);

/*
 * Read fields written by mhit_save (or by the reference's writefield) at
 * iteration t (readfield_restart, multi/readwrite.f90:218-317).  When the
 * sidecar is present the AB2 history is restored; otherwise the next step is
 * Euler with gumax = 1, as in the reference.
 */
int mhit_load(mhit_handle* h, const char* dir, int t);

/*
 * Stand-alone Poisson solve with the step's own kernels: rhs -> p on host
 * arrays (MHIT_LAYOUT_RAW).  Replaces multi/main.f90:732-850 (rhsp ->
 * rhsp_complex -> FFT3D -> divide by -k^2/(nx*ny*nz) -> inverse -> real part),
 * used for the manufactured-solution check of multi/main.f90:739-741, 824-838.
 */
int mhit_poisson(mhit_handle* h, const double* rhs, double* p);

/* Same, on device pointers (raw layout, float64), in the handle's stream. */
int mhit_poisson_device(mhit_handle* h, const double* rhs_dev, double* p_dev);

/* Device pointers of the resident state (raw layout, float64 in the FP64
 * form; float32 in MHIT_FP32_REFINE).  For zero-copy callers; valid until the
 * next mhit_step / mhit_destroy.  u, v, w hold the field BEFORE the pending
 * mean removal; call mhit_sync_state first to materialise it. */
int mhit_device_state(mhit_handle* h, void** u, void** v, void** w, void** phi);

/* Apply the pending mean removal to the resident u, v, w in place. */
int mhit_sync_state(mhit_handle* h);

/* Tile shapes of the stencil kernels: z chunk kz (a divisor of n; 0 = 32)
 * and momentum tile height mty (8 or 16; 0 = the default for n).  Results do
 * not depend on them; the step graphs are re-captured on the next step. */
int mhit_set_tiles(mhit_handle* h, int kz, int mty);

/* Bytes of device memory the handle holds. */
int mhit_memory_bytes(mhit_handle* h, size_t* bytes);

/* Number of kernel launches one step makes (for accounting). */
int mhit_launches_per_step(mhit_handle* h, int* n);

/*
 * Advance `reps` steps with each kernel launched individually between CUDA
 * events on the handle's stream and return the mean duration of every stage
 * in ms[0..*nstages-1] (names from mhit_stage_name).  Same results as
 * mhit_step; used for per-kernel roofline accounting.  The reference times a
 * step with cpu_time (multi/main.f90:332, 948-949) and NVTX ranges
 * (multi/module.f90:61-131).
 */
int mhit_profile_step(mhit_handle* h, int reps, double* ms, int* nstages);
const char* mhit_stage_name(mhit_handle* h, int k);

/* Enqueue nsteps steps without waiting and without reading anything back. */
int mhit_step_async(mhit_handle* h, int nsteps);

/* The handle's CUDA stream (cudaStream_t) and the last CUDA error text. */
void* mhit_stream(mhit_handle* h);
const char* mhit_last_error(mhit_handle* h);

/*
 * Allocation-free Poisson solve (no counterpart in the reference).  For
 * callers that cannot let a library allocate device memory -- an application
 * whose device memory is all owned by its own allocator, or a latency-critical
 * loop that cannot absorb the device-wide synchronisation of cudaFree.  Solves
 * the same problem as mhit_poisson_device (rhs_dev -> p_dev, n^3 float64 on
 * the device, raw layout, k2_mode / grid_mode as in mhit_params) on `stream`
 * (a cudaStream_t, NULL for the default stream), without a handle and without
 * cudaMalloc/cudaFree: its scratch (half spectrum and tables) is a fixed
 * device array of the library for n <= MHIT_NOALLOC_MAX_N (18.9 MB, held on
 * every GPU that loads the library until exit).  Larger n returns
 * MHIT_ERR_SCRATCH_LIMIT.  The first call on a device (with that device
 * current) resolves the scratch address and fills the twiddle and k^2 tables
 * of every supported size with one synchronous host-to-device copy, so make
 * it before any stream capture; later calls only enqueue the solve's kernels
 * on `stream`.  All calls share the scratch: calls that overlap on the GPU
 * race and must be serialised.
 */
#define MHIT_NOALLOC_MAX_N 128
int mhit_poisson_noalloc(const double* rhs_dev, double* p_dev, int n, int k2_mode, int grid_mode,
                         void* stream);

/* ------------------------------------------------------------------------
 * Served ensemble (no counterpart in the reference, which runs one
 * simulation per job).  Independent simulations of uneven grid sizes are
 * queued, admitted as slots and HBM free up (the budget is an HBM-footprint
 * admission limit), kept resident, and advanced together: the simulations of
 * one class (n, precision, phase field, k2_mode, grid_mode) share one CUDA
 * graph of batched kernels that read per-slot arguments from a device table,
 * so admission never re-captures.  Classes run on their own streams.  Each
 * slot computes exactly what mhit_step computes for the same request.
 * ---------------------------------------------------------------------- */
typedef struct mhit_ensemble mhit_ensemble;

#define MHIT_RQ_QUEUED 0
#define MHIT_RQ_RUNNING 1
#define MHIT_RQ_DONE 2
#define MHIT_RQ_FAILED 3
#define MHIT_RQ_CANCELLED 4

typedef struct mhit_ens_info {
  int32_t state;        /* MHIT_RQ_* */
  int32_t status;       /* MHIT_OK or the request's error */
  int32_t n;
  int32_t steps_issued; /* steps enqueued so far */
  double t_submit, t_admit, t_done; /* seconds since mhit_ens_create (-1: not yet) */
  mhit_diag diag;       /* final per-step scalars (done or failed) */
  int32_t kz;           /* the autotuned tile shape of the request's class: stencil z chunk */
  int32_t mty;          /* and momentum tile height */
} mhit_ens_info;

typedef struct mhit_ens_stats_t {
  int64_t rounds, graph_launches;
  size_t bytes_used, bytes_budget;
  int32_t classes, slots;
} mhit_ens_stats_t;

/* mhit_ens_submit flags */
#define MHIT_ENS_KEEP_RESULT 1  /* keep the final fields for mhit_ens_result */
#define MHIT_ENS_BORROW_INPUT 2 /* do not copy u, v, w, phi: the caller keeps them valid and unchanged
                                   until the request is done, failed or cancelled */

/* hbm_budget_bytes = 0: 85% of the free device memory.  Starts the
 * ensemble's transfer threads (host<->device copies of request fields). */
int mhit_ens_create(size_t hbm_budget_bytes, int slots_per_class, mhit_ensemble** out);
/* Queue a request (raw layout float64 inputs, copied unless
 * MHIT_ENS_BORROW_INPUT; flags = MHIT_ENS_* bits). */
int mhit_ens_submit(mhit_ensemble* e, const mhit_params* p, int n, int precision, int phase_field, int nsteps,
                    const double* u, const double* v, const double* w, const double* phi, int flags,
                    int64_t* id);
/* One scheduling round; never waits on the device: publish finished
 * requests, activate uploaded ones, admit what fits, and keep a few
 * milliseconds of batched steps queued on every busy class. */
int mhit_ens_progress(mhit_ensemble* e, int* pending);
/* Sleep until a scheduling round has something to do (a transfer finished,
 * a class has room for more rounds, a request can be retired) or timeout_s
 * passes; *ready = 1 or 0.  A serving loop alternates mhit_ens_progress and
 * mhit_ens_wait instead of spinning on mhit_ens_progress. */
int mhit_ens_wait(mhit_ensemble* e, double timeout_s, int* ready);
int mhit_ens_query(mhit_ensemble* e, int64_t id, mhit_ens_info* out);
/* Final fields of a done request (keep_result = 1), raw layout float64. */
int mhit_ens_result(mhit_ensemble* e, int64_t id, double* u, double* v, double* w, double* phi);
int mhit_ens_release(mhit_ensemble* e, int64_t id);
int mhit_ens_cancel(mhit_ensemble* e, int64_t id);
int mhit_ens_stats(mhit_ensemble* e, mhit_ens_stats_t* out);
const char* mhit_ens_last_error(mhit_ensemble* e);
int mhit_ens_destroy(mhit_ensemble* e);

/* Free everything (multi/main.f90:979-985). */
int mhit_destroy(mhit_handle* h);

/* Text of a status code. */
const char* mhit_strerror(int status);

/* 1 if the grid size has built kernels. */
int mhit_size_supported(int n);

/*
 * Self-check of the bounded wait the stencil kernels use for their staged
 * planes (tensor-map box loads completed on a shared-memory barrier): one
 * warp arms a barrier and waits at most limit_cycles SM clock cycles.  With
 * arrive = 1 a thread arrives and *status_out is MHIT_OK; with arrive = 0
 * nothing arrives, the wait gives up and *status_out is MHIT_ERR_TIMEOUT,
 * the status a step reports when a staged plane never lands.  The kernel
 * returns either way and the CUDA context stays usable.
 */
int mhit_check_bounded_wait(int arrive, long long limit_cycles, int* status_out);

#ifdef __cplusplus
}
#endif

#endif /* MHIT_H */
