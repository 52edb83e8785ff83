/* C ABI of libfvm_b200: the B200 finite-volume residual + Runge-Kutta stage path.
 *
 * The reference (nathanzimniak/multiphysics-fvm) is pure Python/NumPy and has no
 * FFI; these entry points are what its Python surface binds to (by ctypes) when a
 * setup selects this backend.  Each declaration names the reference interface it
 * replaces.  All calls return 0 on success or a negative FVM_E_* code; the message
 * of the last failure on the calling thread is available from fvm_last_error().
 * No C++ exception crosses this boundary.  A handle owns all of its device memory
 * and one CUDA stream; it is not thread-safe, separate handles are independent.
 *
 * Host arrays are float64, C-contiguous, in the reference's own layout: one
 * variable is an (nx1+2, nx2+2, nx3+2) array with one ghost layer
 * (src/physics/navier_stokes.py:33-39); a whole state is (NV, nx1+2, nx2+2, nx3+2)
 * with variables in the reference's allocate_u order.
 */
#ifndef FVM_B200_H
#define FVM_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define FVM_OK 0
#define FVM_E_INVALID (-1)   /* bad argument or unsupported combination (ValueError) */
#define FVM_E_CUDA (-2)      /* CUDA runtime/driver failure */
#define FVM_E_NOMEM (-3)     /* device or pinned allocation failed */
#define FVM_E_STATE (-4)     /* status word non-zero (NaN, rho<=0, P<=0, dt<=0, timeout) */

/* physics (setup["physics"] module) */
#define FVM_NAVIER_STOKES 0
#define FVM_HEAT 1
#define FVM_MAXWELL 2
/* coordinate systems (src/grid/geometry.py:14) */
#define FVM_CARTESIAN 0
#define FVM_CYLINDRICAL 1
#define FVM_SPHERICAL 2
/* space schemes (src/numerics/*.py) */
#define FVM_PIECEWISE_CONSTANT 0
#define FVM_MUSCL 1
#define FVM_MINMOD 0
#define FVM_MONOTONIZED_CENTRAL 1
#define FVM_VAN_LEER 2
#define FVM_RUSANOV 0
#define FVM_HLL 1
/* time integrators (src/numerics/time_integrators.py) */
#define FVM_EULER_EXPLICIT 0
#define FVM_RK3 1
#define FVM_RK3_SSP 2
#define FVM_RK4 3
/* boundary conditions (src/grid/boundary_conditions.py) + Dirichlet (new) */
#define FVM_BC_PERIODIC 0
#define FVM_BC_NEUMANN 1
#define FVM_BC_REFLECTING 2
#define FVM_BC_DIRICHLET 3
/* precision of the device state and stencil arithmetic */
#define FVM_FP32 0
#define FVM_FP64 1
/* status bits (fvm_status) */
#define FVM_ST_NONFINITE 1u
#define FVM_ST_DENSITY 2u
#define FVM_ST_PRESSURE 4u
#define FVM_ST_DT 8u
#define FVM_ST_TIMEOUT 16u

/* Everything a setup dict selects (setups/kelvin_helmholtz.py:154-163).
 * params: navier_stokes {gamma, mu, g1, g2, g3}; heat {rho, cp, k, q};
 *         maxwell {mu, epsilon, sigma, rho_c, chi_B, chi_D}.
 * bc_kind/bc_value: [variable][side], sides ordered left,right,bottom,top,front,back
 * (src/solver.py:36).  tile_ty: tile rows, 0 = the default shape (or the alternative
 * one that fvm_tiling reports after fvm_autotune); zchunk: planes per tile, 0 = 64. */
typedef struct fvm_desc {
  int physics, precision, coords;
  int nx1, nx2, nx3;
  double x1_min, x1_max, x2_min, x2_max, x3_min, x3_max;
  int reconstructor, limiter, riemann, integrator;
  int bc_kind[6][6];
  double bc_value[6][6];
  double params[8];
  int tile_ty, zchunk;
} fvm_desc;

typedef struct fvm_handle fvm_handle;

/* Build the grid + device state for a setup.
 * Replaces geometry.build_grid (src/grid/geometry.py:14-194) and
 * physics.allocate_u (src/physics/navier_stokes.py:13-41) as called by
 * src/solver.py:125-128. */
int fvm_create(const fvm_desc* desc, fvm_handle** out);

/* Release every device/pinned buffer, graph and stream of the handle. */
int fvm_destroy(fvm_handle* h);

/* Number of conserved variables and the device buffer footprint in bytes. */
int fvm_info(const fvm_handle* h, int* nvars, long long* device_bytes);

/* Copy a whole ghosted host state (NV, nx1+2, nx2+2, nx3+2) to the device.
 * Replaces the host-resident U dict written by apply_ics (src/solver.py:64-85). */
int fvm_upload(fvm_handle* h, const double* host_state);

/* Copy the device state back into a ghosted host array (NV, nx1+2, nx2+2, nx3+2).
 * Ghost faces are refreshed from the boundary conditions and ghost edges/corners
 * averaged as in src/solver.py:39-61.  Replaces reading U in io.save_snapshot
 * (src/io.py:14-63). */
int fvm_download(fvm_handle* h, double* host_state);

/* Pipelined transfers: the same copies as fvm_upload / fvm_download (the
 * downloaded ghost edges and corners are averaged on the device, as
 * src/solver.py:39-61), enqueued without waiting.  Uploads run on their own
 * copy stream, downloads on another, so the upload of one step's input, the
 * step (fvm_step_async) and the download of the previous result overlap.  Host
 * buffers should be pinned (pageable memory makes the copy synchronous) and
 * must stay valid and untouched until fvm_synchronize returns.  Replace the
 * host-resident U of src/solver.py:64-85 and io.save_snapshot (src/io.py:14-63)
 * when a caller streams states through the device. */
int fvm_upload_async(fvm_handle* h, const double* host_state);
int fvm_download_async(fvm_handle* h, double* host_state);
/* fvm_step without waiting for the steps to finish (see fvm_step). */
int fvm_step_async(fvm_handle* h, int n_steps, int dt_mode);
/* Wait for everything enqueued on the handle (steps and pipelined copies). */
int fvm_synchronize(fvm_handle* h);

/* dt = CFL / max characteristic rate of the current state, reduced on the device
 * in float64.  Replaces physics.compute_dt (navier_stokes.py:512-585,
 * heat.py:305-351, maxwell.py:533-600). */
int fvm_compute_dt(fvm_handle* h, double cfl, double* dt_out);

/* Residual of the uploaded state exactly as given (ghosts are not refilled),
 * written into host_rhs (NV, nx1, nx2, nx3).  Replaces physics.compute_rhs
 * (navier_stokes.py:588-711, heat.py:354-473, maxwell.py:603-729). */
int fvm_residual(fvm_handle* h, double* host_rhs);

/* Advance n_steps time steps on the device (each step captured once as a CUDA
 * graph: [dt reduction] + per stage {ghost fill, fused stage kernel}).
 * dt_mode 0: dt = compute_dt(cfl) every step, stopping (as no-op steps) once
 * t > t_end (src/solver.py:137-150).  dt_mode 1: the fixed dt of fvm_set_dt.
 * Replaces the time loop body src/solver.py:140-143 and the integrators
 * euler_explicit/rk3/rk3_ssp/rk4 (src/numerics/time_integrators.py:10-221)
 * together with apply_bcs (src/solver.py:13-61). */
int fvm_step(fvm_handle* h, int n_steps, int dt_mode);

/* Same as fvm_step without the final synchronisation of the host, returning the
 * device time of the n_steps graph launches (CUDA events on the handle's stream). */
int fvm_time_steps(fvm_handle* h, int n_steps, int dt_mode, double* ms);

/* Configure the time loop: CFL number, end time (inf = step-counted) and fixed dt. */
int fvm_set_time(fvm_handle* h, double t, double t_end, double cfl);
int fvm_set_dt(fvm_handle* h, double dt);

/* Simulated time, steps taken and the last dt (read back from the device). */
int fvm_get_time(fvm_handle* h, double* t, long long* steps, double* last_dt);

/* Conserved totals sum(U*V) over the interior in float64 with compensated
 * summation (NV values; Maxwell adds the EM energy 0.5(D.E+B.H)V as entry NV).
 * New: the reference has no such diagnostic. */
int fvm_totals(fvm_handle* h, double* totals);

/* Sticky device status word (FVM_ST_* bits); fvm_clear_status resets it. */
int fvm_status(fvm_handle* h, unsigned* status);
int fvm_clear_status(fvm_handle* h);

/* Limit (ns, default 2e9) of every wait of the stage kernels for a plane of
 * the TMA ring or a staged tile.  A wait that runs out sets FVM_ST_TIMEOUT;
 * the block then waits (up to 1 s per copy) for the copies it has in flight
 * and returns, so the context stays usable.  never_complete != 0 is for tests
 * of that path: every ring copy then expects 16 bytes more than it delivers,
 * so no ring wait can complete and each runs out at the limit (the wait for
 * copies in flight is then 0.1 s).  New: the reference has no device waits
 * (its only observability is the print of src/solver.py:147). */
int fvm_set_wait_limit(fvm_handle* h, unsigned long long data_wait_ns, int never_complete);

/* Kernel launches of one fvm_step step (dt_mode as in fvm_step): the CFL
 * reduction (navier_stokes, dt_mode 0), then per stage a ghost fill (the first
 * one also closes the step's clock) and the stage kernel; the closure's
 * kernels (fvm_closure_attach) are not counted. */
int fvm_step_launches(fvm_handle* h, int dt_mode, int* launches);

/* Per-launch device time of the stage kernels (ms, CUDA events on the handle's
 * stream) over n_steps un-captured steps; fills per-stage totals. */
int fvm_profile_steps(fvm_handle* h, int n_steps, int dt_mode, double* stage_kernel_ms,
                      double* other_kernel_ms, int* stage_launches);

/* Pick the block shape -- tile rows (the default and, for float32
 * navier_stokes and heat, a 4-row tile) and the z-march depth (planes per
 * tile) -- by timing every pair on this grid; the state and clock are restored
 * afterwards.  New: the reference has no tuning. */
int fvm_autotune(fvm_handle* h, int* best_zchunk, double* best_ms_per_step);
/* The handle's block shape: tile rows (fvm_desc.tile_ty, or the autotuner's
 * choice) and z-march depth.  New: the reference has no tuning. */
int fvm_tiling(fvm_handle* h, int* tile_ty, int* zchunk);

/* Sharp Kelvin-Helmholtz initial state written on the device (the host
 * initializer of setups/kelvin_helmholtz_sharp.py, done in HBM instead of on
 * the host and uploaded; replaces solver.apply_ics, src/solver.py:64-85, for
 * this setup).  params: {rho_inner, rho_outer, shear_velocity, pressure,
 * amplitude, wavenumber, noise, phase, noise_all}: rho and v1 = +-shear inside /
 * outside |x2 - 0.5| < 0.25, v2 = amplitude*sin(2 pi wavenumber x1 + phase) +
 * noise, v1 and v3 get noise too when noise_all != 0, P = pressure, gamma from
 * the descriptor.  Noise is uniform in [-noise, noise) from a counter-based hash
 * of (seed, variable, cell), so it is reproducible for any grid but is not
 * NumPy's draw.  navier_stokes handles only; ghosts are filled by the step. */
int fvm_init_kelvin_helmholtz(fvm_handle* h, const double params[9], unsigned long long seed);

/* ---- batches of independent grids ----------------------------------------------
 * Many setups of uneven sizes advance together: one persistent launch per kernel
 * specialisation and stage walks a flat tile list over all grids, and every grid
 * keeps its own CFL time step.  All grids share the time integrator and the
 * precision; navier_stokes and heat grids may be mixed.  Each grid is an ordinary
 * handle (fvm_batch_handle) for upload/download/set_time/get_time/totals.
 * Replaces n independent solver.run loops (src/solver.py:88-151). */
typedef struct fvm_batch fvm_batch;
int fvm_batch_create(const fvm_desc* descs, int n, fvm_batch** out);
int fvm_batch_destroy(fvm_batch* b);
int fvm_batch_size(const fvm_batch* b, int* n, long long* tiles);
int fvm_batch_handle(fvm_batch* b, int i, fvm_handle** h);
int fvm_batch_step(fvm_batch* b, int n_steps, int dt_mode);
int fvm_batch_time_steps(fvm_batch* b, int n_steps, int dt_mode, double* ms);
/* Times the batch over z-march depths (and, for a mixed launch with heat grids,
 * the heat tiles' heights, 20 or 10 rows) on the live states, restores them and
 * keeps the fastest; fvm_tiling on a member handle reports its tile rows. */
int fvm_batch_autotune(fvm_batch* b, int* best_zchunk, double* best_ms_per_step);
/* Kernel launches per Runge-Kutta stage of one batched step.  It is 1 when every
 * grid is float32 and either inviscid cartesian navier_stokes (one limiter and
 * Riemann solver) or piecewise-constant heat (one coordinate system): those run
 * as one mixed launch.  Other batches launch once per kernel specialisation. */
int fvm_batch_launches(const fvm_batch* b, int* per_stage);

/* Conserved totals sum_q(cells[q][i] * volumes[i]) in float64 with compensated
 * summation, computed without allocating any device memory.  No counterpart in
 * the reference.  For callers that cannot call cudaMalloc (a host framework
 * that owns every allocation, an embedded runtime that forbids allocation
 * after start-up): the per-block partial sums live in a fixed 64 KiB device
 * array inside the library, which every GPU that loads the library holds
 * until the process exits.  cells: float32 device array (nvars, ncells), any
 * cell order; volumes: float64 device array (ncells); totals: float64 device
 * array of nvars outputs.  nvars must be 1..8 (FVM_E_INVALID otherwise).  Work
 * is enqueued on `stream` (a cudaStream_t, 0 = legacy default stream) and not
 * waited for.  The first call on a device (with that device current) resolves
 * the array's device address and keeps it for the process; that address
 * belongs to the device's primary context, so it is not valid after
 * cudaDeviceReset or in another driver-API context.  Make the first call
 * before any stream capture.  All calls
 * share the one array: calls whose kernels can overlap on the GPU (other
 * streams, other host threads) race and must be serialised by the caller. */
int fvm_totals_noalloc(const float* cells, const double* volumes, int nvars, long long ncells, double* totals,
                       void* stream);

/* Copy the message of the last failure on this thread into buf. */
int fvm_last_error(char* buf, int len);

#ifdef __cplusplus
}
#endif
#endif /* FVM_B200_H */
