/*
 * ymkh.h — C ABI of the B200-native Kelvin–Helmholtz step of the 2D two-fluid
 * SU(2) Yang–Mills simulator (drop-in for the step loop of ymgpu2d).
 *
 * The reference has no plugin API: the unit this library replaces is the body
 * of the time loop in ymgpu2d/main_ym.cu:322-479, which operates on the SoA
 * pointer structs YMFieldPtrs / YMFluidPtrs (ymgpu2d/YM_Physics.cuh:11-29)
 * and YMParams (ymgpu2d/YM_Physics.cuh:31-46) on the legacy default stream.
 *
 * Conventions
 *  - Every array is NX*NZ FP64, x (shear axis) fastest: idx = x + z*NX
 *    (ymgpu2d/FCT_DeviceMath.cuh:12).  The caller owns the state; the library
 *    owns only small internal tables and, for the batched entry points, a run
 *    table.
 *  - State order (24 arrays) used by every entry point:
 *      fields[12] = Ex1 Ex2 Ex3 Ez1 Ez2 Ez3 By1 By2 By3 Az1 Az2 Az3
 *      fluidA[6]  = n px pz Q1 Q2 Q3          (beam A, +z)
 *      fluidB[6]  = n px pz Q1 Q2 Q3          (beam B, -z)
 *    The reference's derived arrays (ux, uy, J, sources, E_therm, transposed
 *    and padded copies) are not state: they are recomputed inside the fused
 *    kernels from the arrays above.
 *  - Return codes: 0 = ok, negative = error (YMKH_E*); the message of the last
 *    error on the calling thread is available from ymkh_last_error().  No C++
 *    exception crosses this boundary.
 *  - Streams: `stream` is a cudaStream_t passed as void*; NULL = legacy
 *    default stream (what the reference uses).  Every call is stream-ordered;
 *    only the calls with host results (ymkh_energy, ymkh_mode_amp,
 *    ymkh_circ_amp, ymkh_gauss, ymkh_check) synchronise the stream.
 *  - Threading: one context per host thread at a time.
 */
#ifndef YMKH_H
#define YMKH_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define YMKH_NFIELDS 12
#define YMKH_NFLUID 6
#define YMKH_NSTATE 24
#define YMKH_MAX_EXTRA_BANDS 4

enum {
  YMKH_OK = 0,
  YMKH_EINVAL = -1,   /* bad argument / unsupported size */
  YMKH_ECUDA = -2,    /* CUDA runtime error */
  YMKH_ESTATE = -3,   /* state not bound / context misuse */
  YMKH_ENOMEM = -4    /* allocation failed */
};

/* Forms of the flux-corrected transport stage (same results bit for bit):
 * FUSED streams x- and z-sweeps in one pass (fewest bytes, staged rows);
 * SPLIT runs a coalesced x pass into a 12-array scratch and a coalesced
 * z pass (more bytes, full-bandwidth access). */
enum { YMKH_FCT_FUSED = 0, YMKH_FCT_SPLIT = 1 };

/* Filter engines for the periodic-direction DFT mode filter. */
enum {
  YMKH_FILTER_DFT = 0,   /* dense DFT with the reference's FP32-phase twiddles, FP64 sums
                            (ymgpu2d/YM_Physics.cu:349-584) */
  YMKH_FILTER_TF32X3 = 1 /* the same two contractions on the tensor cores: operands split
                            into TF32 hi + lo, three passes, FP32 accumulation (a precision
                            change confined to the subtracted band).
                            No reference counterpart. */
};

/* GridParams (ymgpu2d/FCT_DeviceMath.cuh:14-17): ny/dy of the reference are
 * the periodic z axis here. */
typedef struct ymkh_grid {
  int nx, nz;
  double dx, dz;
} ymkh_grid;

/* YMParams (ymgpu2d/YM_Physics.cuh:31-46), field for field, followed by the
 * extensions this library adds.  Derivation from the .ini keys follows
 * ymgpu2d/main_ym.cu:51-83. */
typedef struct ymkh_params {
  double dx, dz, dt_step;
  double c, eps_0;
  double alpha_YM;
  double V0, epsilon;
  int freeze_az1;         /* skip Az1 update */
  int periodic_x;         /* periodic shear axis (run_mode >= 1) */
  double xi_sponge;       /* 0 = off */
  double sigma_sponge;
  double xi_cut;          /* 0 = off */
  double warm_T;          /* isothermal closure, 0 = cold */
  int suppress_kz0;       /* z-mean removal + colour-1 EM zeroing */
  double hyp_diff_coeff;  /* 4th-order z hyperdiffusion, 0 = off */
  int kz_suppress_max;    /* band 1 = [1, kz_suppress_max] when >= 1 */
  int kz_suppress_hi;     /* band 2 = [kz_suppress_max+2, kz_suppress_hi] when > max+1 */
  /* --- extensions (not in the reference) --- */
  int n_extra_bands;      /* further bands [lo, hi], applied after the two above */
  int extra_band_lo[YMKH_MAX_EXTRA_BANDS];
  int extra_band_hi[YMKH_MAX_EXTRA_BANDS];
  int filter_engine;      /* YMKH_FILTER_* */
} ymkh_params;

/* Arguments of kernel_ym_init (ymgpu2d/YM_Init.cu:32-40, YM_Init.cuh:10-17).
 * Seed profiles are HOST arrays of nx doubles (already interpolated to the
 * grid, as ymgpu2d/main_ym.cu:198-206 does) or NULL. */
typedef struct ymkh_init_params {
  int run_mode;
  int k_mode;
  double perturb_amp;
  double V0;
  double epsilon;
  double alpha_YM;
  int init_by1_eq;
  double vz_edge_taper;
  const double* seed_by;
  const double* seed_ex;
  const double* seed_ez;
  const double* seed_az;
  const double* seed_qA;
  const double* seed_qB;
} ymkh_init_params;

typedef struct ymkh_ctx ymkh_ctx;

/* Copies the last error message of the calling thread into buf (NUL
 * terminated, truncated to n).  Returns the last error code. */
int ymkh_last_error(char* buf, size_t n);

/* Replaces the allocation/derivation block of ymgpu2d/main_ym.cu:63-121:
 * validates sizes (the reference's constraints of ymgpu2d/YM_Config.cu:203-211
 * are checked by the caller's config layer; here only what the kernels need),
 * builds the FP32-phase twiddle table on the device. */
int ymkh_create(const ymkh_grid* grid, const ymkh_params* params, ymkh_ctx** out);

/* Updates the step parameters of an existing context (same grid). */
int ymkh_set_params(ymkh_ctx* ctx, const ymkh_params* params);

/* Binds caller-owned device arrays (YMFieldPtrs / YMFluidPtrs without the
 * derived arrays).  Pointers must stay valid until rebound or destroyed. */
int ymkh_bind_state(ymkh_ctx* ctx, double* const fields[YMKH_NFIELDS],
                    double* const fluidA[YMKH_NFLUID], double* const fluidB[YMKH_NFLUID]);

/* Zero-copy double buffering: the fused kernels read start-of-step values
 * of neighbouring tiles, so each step writes a second 24-array set.  With
 * ymkh_bind_state the library allocates that set and copies back when a call
 * ends on it; with ymkh_bind_state2 the caller provides both sets (24
 * pointers each, state order) and reads the current one from
 * ymkh_current_buffer().  No reference counterpart (the reference copies the
 * fluid state four times per step, ymgpu2d/YM_Fluid.cu:134-143). */
int ymkh_bind_state2(ymkh_ctx* ctx, double* const* state0, double* const* state1);
int ymkh_current_buffer(ymkh_ctx* ctx);
int ymkh_set_current_buffer(ymkh_ctx* ctx, int which);

/* Launch-shape controls used by the autotuner: steps per captured CUDA graph
 * (even, 0 = no graphs) and the FCT strip width (32/64/128) and z-segment
 * length (the unit of work that CTAs share out; each CTA runs a contiguous
 * block of segments).  No reference counterpart. */
int ymkh_set_graph_steps(ymkh_ctx* ctx, int nsteps_per_graph);
int ymkh_set_fct_shape(ymkh_ctx* ctx, int strip_width, int segment_rows);
int ymkh_get_fct_shape(ymkh_ctx* ctx, int* strip_width, int* segment_rows);
int ymkh_set_fct_mode(ymkh_ctx* ctx, int mode);  /* YMKH_FCT_* (default FUSED); the autotuner picks per size class */

/* Device time per stage over nsteps uncaptured steps (CUDA events between
 * stages on `stream`), accumulated in out_ms[0..6]: FCT, Maxwell,
 * sponge/xi_cut, z-mean, band filters, hyperdiffusion, colour-1 zeroing.
 * nout must be >= 7.  No reference counterpart. */
int ymkh_stage_times(ymkh_ctx* ctx, int nsteps, void* stream, float* out_ms, int nout);

/* kernel_ym_init (ymgpu2d/YM_Init.cu:32-257) on the bound state; the
 * velocity/source precompute of ymgpu2d/main_ym.cu:228-237 is not needed
 * because sources are recomputed inside ymkh_step. */
int ymkh_init(ymkh_ctx* ctx, const ymkh_init_params* ip, void* stream);

/* nsteps iterations of ymgpu2d/main_ym.cu:324-455 (stages 1-7) on the bound
 * state, in the reference's stage order. */
int ymkh_step(ymkh_ctx* ctx, int nsteps, void* stream);

/* Total energy of ymgpu2d/YM_Energy.cu:3-32 (per-cell energy summed over the
 * grid; here a fixed-order compensated device reduction).  The _async form
 * writes one double to device memory without synchronising. */
int ymkh_energy(ymkh_ctx* ctx, double* host_out, void* stream);
int ymkh_energy_async(ymkh_ctx* ctx, double* dev_out, void* stream);

/* Mode amplitude of ymgpu2d/analysis/remote_timeseries.py:62-77:
 * out[0] = mean_x |sum_z (Az2 + i Az3) e^{-2 pi i k z / NZ}| / NZ,
 * out[1] = the same for the conjugate signal (Az2 - i Az3). */
int ymkh_mode_amp(ymkh_ctx* ctx, int k, double* host_out2, void* stream);

/* Colour-2/3 pairs of ymkh_circ_amp. */
enum { YMKH_PAIR_AZ = 0, YMKH_PAIR_BY = 1, YMKH_PAIR_EX = 2, YMKH_PAIR_EZ = 3 };

/* Circular mode amplitude of a colour-2/3 pair (F2 + i F3, F one of Az, By,
 * Ex, Ez) at wavenumber k along z.  With host_weight NULL, the x-mean of
 * ymkh_mode_amp; with NX weights, out[0] = sum_x w[x] |F_k(x)| / NZ and out[1]
 * the same for F2 - i F3: the shear-layer weighted amplitude of
 * ymgpu2d/analysis/resolution_convergence.py:77-86 (there from CSV snapshots,
 * with w = sech((x - LX/2)/EPS) normalised).  Synchronises `stream`. */
int ymkh_circ_amp(ymkh_ctx* ctx, int pair, int k, const double* host_weight, double* host_out2, void* stream);

/* Non-Abelian Gauss law G^a = dEx^a/dx + dEz^a/dz + alpha (Az x Ez)^a - rho^a
 * of ymgpu2d/analysis/gauss_check.py:40-110 (offline there, from CSV
 * snapshots), on the current state: Yee differences with periodic wrap in x
 * and z, Ez averaged to the cell centre, rho^a = Q^a_A nA + Q^a_B nB, and the
 * state's own Az1.  host_out receives YMKH_GAUSS_NOUT root-mean-squares over
 * the grid: [0..2] G^a, [3..5] div E^a, [6..8] alpha (Az x Ez)^a,
 * [9..11] rho^a, [12..14] div E^a + alpha (Az x Ez)^a, [15] |Ex1|+..+|Ez3|.
 * Synchronises `stream`. */
#define YMKH_GAUSS_NOUT 16
int ymkh_gauss(ymkh_ctx* ctx, double* host_out, void* stream);

/* Snapshots of the current state (ymgpu2d/main_ym.cu:260-313).  The call
 * enqueues the device-to-host copies on `stream` and returns; a writer
 * thread waits for them and writes the file, at most 4 writers at a time
 * (the oldest is joined first, as in the reference).
 *  YMKH_SNAP_CSV:  the reference's 26-column CSV, byte for byte: header
 *                  X,Z,By1,By2,By3,Az2,Az3,PzA,PxA,Q1A,PzB,PxB,Q1B,Ex1,Ex2,Ex3,
 *                  Ez1,Ez2,Ez3,nA,nB,Q2A,Q3A,Q2B,Q3B,Az1; rows z-major, x
 *                  fastest; X = x*dx, Z = z*dz; every value as printf "%g".
 *  YMKH_SNAP_FP64: exact binary: a 40-byte header (char[8] "YMKHSNP1",
 *                  uint32 version 1, nx, nz, narrays = 24, double dx, dz)
 *                  then the 24 arrays in state order, native byte order.
 * The copies read the state at their place in `stream`'s order: work that
 * changes the state on another stream must wait for `stream`.  Errors of a
 * writer (file cannot be opened or written) are returned by the next
 * ymkh_snapshot or ymkh_snapshot_wait.  ymkh_destroy waits too. */
enum { YMKH_SNAP_CSV = 0, YMKH_SNAP_FP64 = 1 };
int ymkh_snapshot(ymkh_ctx* ctx, const char* path, int format, void* stream);
int ymkh_snapshot_wait(ymkh_ctx* ctx);

/* Reports (and clears) the device error word: YMKH_ECUDA if a bounded wait
 * inside a kernel timed out (a staged row that never arrived,
 * YMKH_ERR_WAIT) or, in the debug build, an out-of-range access was skipped
 * (YMKH_ERR_BOUNDS) since the last check.  Synchronises `stream`;
 * ymkh_energy calls it.  No reference counterpart. */
int ymkh_check(ymkh_ctx* ctx, void* stream);

/* Frees the context (not the bound state). */
int ymkh_destroy(ymkh_ctx* ctx);

/* The reference's FP32 filter twiddles (ymgpu2d/YM_Physics.cu:387-388)
 * evaluated on the current device for modes [m_lo, m_hi] and z in [0, nz):
 * cos_out/sin_out are host arrays of (m_hi-m_lo+1)*nz floats, mode-major. */
int ymkh_twiddles(int nz, int m_lo, int m_hi, float* cos_out, float* sin_out);

/* Batches (no reference counterpart; the reference runs one configuration
 * per process, ymgpu2d/scripts/*.sh).  Bound runs of any grid sizes and
 * parameters advance together: each step launches one FCT and one Maxwell
 * kernel over the (run, strip, segment) items of all members, then the
 * per-run filter stages.  A run's state after k batch steps is bit-identical
 * to k ymkh_step calls on it alone.  Membership may change between calls
 * (continuous batching); a run belongs to at most one batch at a time and
 * must not be stepped alone while it is a member. */
typedef struct ymkh_batch ymkh_batch;
int ymkh_batch_create(ymkh_batch** out);
int ymkh_batch_add(ymkh_batch* batch, ymkh_ctx* run);
int ymkh_batch_remove(ymkh_batch* batch, ymkh_ctx* run);
int ymkh_batch_size(ymkh_batch* batch);
int ymkh_batch_set_graph_steps(ymkh_batch* batch, int nsteps_per_graph);
int ymkh_batch_set_fct_mode(ymkh_batch* batch, int mode);
int ymkh_batch_step(ymkh_batch* batch, int nsteps, void* stream);
int ymkh_batch_check(ymkh_batch* batch, void* stream);
int ymkh_batch_destroy(ymkh_batch* batch);

/* Number of kernel launches issued by this library since load (all entry
 * points, all threads).  Used to report launch counts. */
long long ymkh_launch_count(void);

/* How the loaded library was built (no reference counterpart): a bit set of
 * YMKH_BUILD_DEBUG, set in libymkh_debug.so, whose fused kernels check every
 * global row copy and store against its array before making it; a failed
 * check skips the access and sets YMKH_ERR_BOUNDS in the error word that
 * ymkh_check / ymkh_batch_check report.  Nothing traps. */
#define YMKH_BUILD_DEBUG 1
#define YMKH_ERR_WAIT 1u   /* error word: a bounded in-kernel wait ran out */
#define YMKH_ERR_BOUNDS 2u /* error word (debug build): an out-of-range access was skipped */
int ymkh_build_flags(void);

/* Total energy of a caller-bound state without any device allocation by the
 * library (no context; no reference counterpart: the reference sums energy
 * through a buffer it allocates, ymgpu2d/YM_Energy.cu:23-32).  For callers
 * that cannot allow cudaMalloc: an arena that owns the device memory, a
 * multi-stream loop that must not be synchronised by allocation, or code
 * holding only the 24 state arrays.  Same kernels and summation order as
 * ymkh_energy_async, so the same total bit for bit.  state: 24 device
 * pointers in state order; writes one double to dev_out on `stream`.
 * Partial sums live in a static device array sized for at most
 * YMKH_NOALLOC_MAX_CELLS cells; larger grids return YMKH_EINVAL.  The first
 * call on each device (that device current) looks up the array's address
 * (cudaGetSymbolAddress) and caches it: make it before any stream capture.
 * The cache is per device and assumes the device's primary context (the
 * runtime's): it is not valid under a caller's own driver-API context, nor
 * across cudaDeviceReset. 
 * Calls that overlap on one device share the array and race: keep them on
 * one stream or one after another. */
#define YMKH_NOALLOC_MAX_CELLS 134217728
int ymkh_energy_noalloc(double* const* state, int nx, int nz, double* dev_out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* YMKH_H */
