/*
 * pysweep_b200 -- C ABI of the B200 swept space-time solver.
 *
 * One ps_solver owns the device state of one periodic 2-D field
 * ([nv][nx][ny] doubles, C order, the reference's (v, x, y) layout without
 * the time axis), the buffers the swept and standard decompositions need, and
 * one CUDA stream.  Calls on one solver are serialised by the caller; solvers
 * on different host threads are independent.  Every entry point returns
 * PS_OK (0) or a negative PS_ERR_* code; nothing aborts the process and no
 * call blocks on the device unless its description says so.  Host pointers
 * are borrowed for the duration of the call only.
 *
 * Each declaration names the reference interface it replaces (paths relative
 * to the anthony-walker/pysweep checkout).
 */
#ifndef PYSWEEP_B200_H
#define PYSWEEP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define PS_OK 0
#define PS_ERR_INVALID (-1)     /* bad argument or configuration */
#define PS_ERR_CUDA (-2)        /* a CUDA runtime/driver call failed */
#define PS_ERR_NOMEM (-3)       /* device allocation failed */
#define PS_ERR_TIMEOUT (-4)     /* a bounded device-side wait gave up */
#define PS_ERR_UNSUPPORTED (-5) /* configuration this build does not provide */
#define PS_ERR_COMPILE (-6)     /* a user step hook failed to compile */
#define PS_ERR_STATE (-7)       /* call out of order (e.g. run before set_state) */

/* built-in equations (the reference's plugins, pysweep/equations/*.py + *.cu) */
#define PS_EQ_HEAT 0
#define PS_EQ_EULER 1
#define PS_EQ_EXAMPLE 2
#define PS_EQ_CHECKER 3
#define PS_EQ_HALF 4
/* Heat with a courant number per cell (one variable) and its adjoint, the
 * kernels of the differentiable solve (pysweep_b200.adjoint): in lambda (two
 * variables: lambda and the accumulated dJ/dC) or in mu = C .* lambda (one
 * variable; the sum of mu .* L(u) accumulates in grid field 2).  Their grid
 * fields are set with ps_set_field. */
#define PS_EQ_HEATVAR 6
#define PS_EQ_HEATVAR_ADJ 7
#define PS_EQ_HEATVAR_ADJMU 8

/* Storage type of a solver's fields (ps_create_typed).  PS_DTYPE_F32 is the
 * reference's `dtype: float32` (pysweep/core/io.py:72-73): every level is
 * stored in float32 and evaluated in float64 (the plugin's constants are
 * float64 scalars), i.e. rounded to float32 once per level.  Heat with
 * forward Euler only. */
#define PS_DTYPE_F64 0
#define PS_DTYPE_F32 1

/* decompositions (yaml key "swept", pysweep/core/io.py:46) */
#define PS_MODE_SWEPT 0
#define PS_MODE_STANDARD 1

typedef struct ps_solver ps_solver;

/*
 * Create a solver for an nv x nx x ny periodic field.
 * Replaces the device half of block.sweptBlock/standardBlock
 * (pysweep/core/block.py:21-43, 64-104, 193-213): context creation,
 * GPU array allocation and the framework constants of io.copyConstants
 * (pysweep/core/io.py:169-184).  ops = stencil half-width ("operating_points"),
 * its = intermediate stages ("intermediate_steps"), blocksize = bs
 * (MPSS = bs/(2*ops) - 1, pysweep/core/solver.py:119).
 */
int ps_create(ps_solver **out, int device, int equation, int nv, int nx, int ny, int ops, int its,
              int blocksize);

/* ps_create with the fields' storage type (PS_DTYPE_F64 or PS_DTYPE_F32; the
 * yaml key `dtype`, pysweep/core/io.py:72-73).  With PS_DTYPE_F32 every
 * buffer passed to ps_set_state, ps_get_state, ps_get_rows, ps_set_rows and
 * ps_run's frames holds floats (the `double *` parameters are then read as
 * `float *`). */
int ps_create_typed(ps_solver **out, int device, int equation, int nv, int nx, int ny, int ops,
                    int its, int blocksize, int dtype);

/*
 * Create a solver whose step function is a user hook compiled at run time:
 * `source` is the text of a plugin's .cu file that defines
 *     __device__ void step(double *shared_state, int idx, int globalTimeStep)
 * and its own __device__ __constant__ globals, exactly as the reference's
 * plugins do (pysweep/equations/*.cu); `name` labels it in compiler messages.
 * Replaces io.buildGPUSource (pysweep/core/io.py:146-155), which includes the
 * file into pysweep.cu (pysweep/core/pysweep.cu:25) and builds it with PyCUDA.
 * The hook sees the framework constants of pysweep/core/pysweep.cu:12-20 (VARS,
 * TIMES, MPSS, MOSS, NV, OPS, ITS, SX, SY): variable v of its cell is
 * shared_state[idx + v*VARS], the neighbours are idx +- SY (x, rows) and
 * idx +- 1 (y, columns) up to OPS away, the previous level is idx - TIMES
 * (its own cell only) and it writes the next level at idx + TIMES.  It is
 * compiled with NVRTC for sm_100a with --fmad=false (every operation rounded
 * separately); the swept and standard decompositions run the same compiled
 * hook, so their results are bitwise equal.  Its constants are set by name
 * with ps_set_global (the value is converted to the declared type).  On a
 * compiler error the call returns PS_ERR_COMPILE and ps_last_error(NULL)
 * holds the compiler's log.  nv in 1..8, ops in 1..4, its in 1..2; fields are
 * float64.  The levels per half-cycle default to MPSS, or fewer where the
 * tiles of one level per slot would not fit in shared memory.
 */
int ps_create_hook(ps_solver **out, int device, const char *source, const char *name, int nv,
                   int nx, int ny, int ops, int its, int blocksize);

/*
 * Compile a step hook without a device (the check io.buildGPUSource's
 * SourceModule performs at Solver start, pysweep/core/io.py:146-155): PS_OK, or
 * PS_ERR_COMPILE with the compiler's log in `log` (loglen bytes at most).
 */
int ps_hook_check(const char *source, const char *name, int nv, int ops, int its, char *log,
                  size_t loglen);

/* Release everything the solver owns.  Replaces process.cleanupProcesses'
 * context pop (pysweep/core/process.py:28-33). */
int ps_destroy(ps_solver *s);

/*
 * Set a named plugin constant (e.g. "DT", "DX", "DY", "ALPHA", "SCHEME",
 * "GAMMA", "GAM_M1", "DTDX", "DTDY").  Replaces
 * source_mod.get_global(name) + cuda.memcpy_htod(ptr, value) in the plugins'
 * set_globals (pysweep/equations/heat.py:38-46, euler.py:25-31).  nbytes is
 * 8 for a double, 4 for an int32, 1 for a bool; the value is converted to the
 * constant's type.
 */
int ps_set_global(ps_solver *s, const char *name, const void *value, size_t nbytes);

/*
 * Look up a named constant: *size receives its size in bytes and *handle an
 * opaque handle usable with ps_set_global_handle.  Framework constants
 * (NV, SX, SY, VARS, TIMES, MPSS, MOSS, OPS, ITS; pysweep/core/pysweep.cu:12-20)
 * are readable through ps_get_global_value.  Replaces
 * SourceModule.get_global (pysweep/equations/heat.py:43).
 */
int ps_get_global(ps_solver *s, const char *name, void **handle, size_t *size);
int ps_set_global_handle(ps_solver *s, void *handle, const void *value, size_t nbytes);
int ps_get_global_value(ps_solver *s, const char *name, double *value);

/*
 * Tiling knobs of the swept decomposition (0 keeps the current value):
 * h = levels per half-cycle (1..MPSS), nseg = column blocks per row band,
 * chunk = streaming chunk width (32 or 64) of the generic streams,
 * threads = 128 (default: register-resident heat streams where they apply)
 * or 256 (always the generic shared-memory streams).
 * The defaults reproduce the reference's bs-row bands with MPSS levels per
 * half-cycle, except heat with forward Euler at bs 32 (12 levels, measured
 * faster); results do not depend on the tiling.
 */
int ps_configure(ps_solver *s, int h, int nseg, int chunk, int threads);

/*
 * The tiling in use: levels per half-cycle, column blocks per band (after a
 * swept run, the count it chose), chunk width and MPSS (bs/(2*OPS) - 1, the
 * most levels a half-cycle can hold).  Any pointer may be NULL.  No
 * counterpart in the reference, whose half-cycle is always MPSS levels
 * (pysweep/core/solver.py:113-128).
 */
int ps_get_tiling(ps_solver *s, int *h, int *nseg, int *chunk, int *mpss);

/*
 * Upload the initial condition.  src holds `levels` fields of nv*nx*ny
 * doubles, oldest first; with levels == 1 the field is copied to every base
 * level, as sweptBlock/standardBlock fill sharedArray[i] for i < ITS
 * (pysweep/core/block.py:24-25, 218-221).  src_on_device != 0 means src is a
 * device pointer.  Replaces the memcpy_htod of the GPU window
 * (pysweep/core/functions.py:21-22).
 */
int ps_set_state(ps_solver *s, const double *src, int levels, int src_on_device);

/*
 * Advance nlevels levels (nlevels = steps * its).  The level computed first is
 * seen by the step function as globalTimeStep = gts0 (the reference starts at
 * 1, pysweep/core/solver.py:162).  If frames != NULL, every frame_every-th
 * completed full step k (k % its == 0 levels) is stored at
 * frames[k/frame_every - 1] ([frame_cap][nv][nx][ny]), the levels
 * io.sweptWrite/standardWrite select (pysweep/core/io.py:134-144, 186-208);
 * frames_on_device != 0 means frames is a device pointer (else the copies go
 * through the solver's stream and the call returns after they land).
 * Replaces solver.sweptSolve / standardSolve (pysweep/core/solver.py:158-189)
 * with the phase sequence FirstPrism/UpPrism/LastPrism
 * (pysweep/core/functions.py:12-88) and Geometry.callGPU
 * (pysweep/core/geometry.py:38-46).  Asynchronous with respect to the host
 * when frames is NULL or on the device.
 */
int ps_run(ps_solver *s, int mode, int64_t nlevels, int gts0, double *frames, int64_t frame_cap,
           int frame_every, int frames_on_device);

/*
 * Grid fields of PS_EQ_HEATVAR and PS_EQ_HEATVAR_ADJ solvers ([nx][ny] device
 * arrays the caller keeps alive while runs are queued).  index 0: courant
 * numbers alpha*dt/dx^2 (both equations).  index 1: an array of
 * [LEN][nx][ny] (LEN: the solver's constant of that name, ps_set_global); for
 * PS_EQ_HEATVAR (NULL allowed) it receives, for every level gts a run
 * computes, the old level's Laplacian at index gts-1; PS_EQ_HEATVAR_ADJ and
 * PS_EQ_HEATVAR_ADJMU (a checkpoint segment of LEN steps, walked backward)
 * read the Laplacian of level gts at index LEN-gts.  index 2
 * (PS_EQ_HEATVAR_ADJMU): the [nx][ny] sum of mu_{n+1} .* L(u_n), updated in
 * place.  ps_run refuses runs whose levels gts0 .. gts0+nlevels-1 fall
 * outside 1 .. LEN.  No C-ABI counterpart in the reference (its solver has no
 * adjoint).
 */
int ps_set_field(ps_solver *s, int index, double *d_field);

/* Copy base level `level` (0 = newest, 1 = the one before) to dst.
 * Replaces the memcpy_dtoh after each phase group (functions.py:32). */
int ps_get_state(ps_solver *s, double *dst, int level, int dst_on_device);

/* Copy rows [row0, row0+nrows) of every variable of base level `level`
 * (0 = newest) to / from a packed [nv][nrows][ny] buffer.  These move the
 * edge strips of a row slab between ranks after each swept half-cycle:
 * they replace the numpy copy of the last/first `splitx` rows that
 * sendForward / sendBackward hand to MPI Sendrecv and write back into the
 * shared array (pysweep/core/functions.py:101-123, rows split among ranks in
 * pysweep/core/process.py:131-176).  Host buffers make the call blocking. */
int ps_get_rows(ps_solver *s, int level, int row0, int nrows, double *dst, int dst_on_device);
int ps_set_rows(ps_solver *s, int level, int row0, int nrows, const double *src,
                int src_on_device);

/* Wait for all work queued on the solver's stream; returns the first device
 * error seen (PS_ERR_TIMEOUT when a bounded wait gave up). */
int ps_synchronize(ps_solver *s);

/* Use the given cudaStream_t (NULL = the solver's own stream). */
int ps_set_stream(ps_solver *s, void *stream);

/*
 * Per-kernel device timing.  ps_profile(s, 1) resets the counters and brackets
 * every following launch with CUDA events on the solver's stream;
 * ps_profile_read returns, for one kernel kind (0 prism stream, 1 Y-bridge
 * seam, 2 gap stream, 3 octahedron seam, 4 standard step), the summed device
 * time in ms, the number of launches and the algorithmic cell updates those
 * launches performed.  Both synchronise the stream.  No reference
 * counterpart: the reference times whole runs only (pysweep/core/io.py:10-27).
 */
int ps_profile(ps_solver *s, int enable);
int ps_profile_read(ps_solver *s, int kind, double *ms, int64_t *launches, double *cells);

/* Kernels launched by this solver so far (all entry points together). */
int64_t ps_kernel_launches(const ps_solver *s);

/* Last error message of this solver (never NULL); with s == NULL, the message
 * of the last failed ps_create on this thread. */
const char *ps_last_error(const ps_solver *s);

/*
 * Swept heat solve (forward Euler, the heat plugin's arithmetic) that
 * allocates nothing.  No counterpart in the reference: it exists for callers
 * that cannot call cudaMalloc at the time they solve -- a process whose memory
 * pool already owns the device memory, a real-time loop that must not touch
 * the allocator.  The caller
 * passes the input and output fields (device pointers, nx*ny doubles, not
 * overlapping each other or the scratch array; overlaps are rejected);
 * every temporary lives in one static device array of 128 MiB that each GPU
 * holds from library load to process exit.  Sizes whose scratch (one field plus
 * the prism faces, about 22*nx*ny bytes at blocksize 32) exceeds it are
 * rejected with PS_ERR_INVALID and a message in err.  The first call on a
 * device resolves the array's device address, so make it before any stream
 * capture; that address is kept for the life of the process, so a
 * cudaDeviceReset after the first call is not supported.  Calls share the array: two calls that overlap on the GPU (other
 * streams, other host threads) race and corrupt each other.  No part of the
 * array needs to start at zero (every half-cycle writes what it reads).
 * Computes nsteps steps of courant = alpha*dt/dx/dx on `stream` (NULL = the
 * default stream); blocksize 16 or 32, nx a multiple of it, ny of 64.
 */
int ps_heat_swept_noalloc(const double *d_in, double *d_out, int nx, int ny, int blocksize,
                          int64_t nsteps, double alpha, double dt, double dx, void *stream,
                          char *err, size_t errlen);

/*
 * Batches: many independent fields (uneven sizes, one equation, one blocksize)
 * advanced together.  No counterpart in the reference, which runs one field
 * per Solver; the per-instance equivalent is one ps_solver per field.  Every
 * phase of a half-cycle is one launch for all instances (a flat table of
 * (instance, band segment) units); with use_graph != 0 the launches of a whole
 * run are captured once into a CUDA graph and replayed.  Constants are per
 * instance (index) or for all (index = -1).  Each instance counts the levels
 * run since its state was set: the first level after ps_batch_set_state sees
 * globalTimeStep = 1 (pysweep/core/solver.py:162) and consecutive
 * ps_batch_run calls continue the count, so runs of any length (odd ones with
 * two stages included) add up to one run of their total.  Register streams (heat, forward
 * Euler, blocksize 16/32) need nx, ny multiples of 32; the other equations use
 * the shared-memory streams with one segment per band.
 */
typedef struct ps_batch ps_batch;
int ps_batch_create(ps_batch **out, int device, int equation, int count, const int *nx,
                    const int *ny, int nv, int ops, int its, int blocksize);
int ps_batch_destroy(ps_batch *b);
int ps_batch_set_global(ps_batch *b, int index, const char *name, const void *value,
                        size_t nbytes);
int ps_batch_set_state(ps_batch *b, int index, const double *src, int levels, int src_on_device);
int ps_batch_run(ps_batch *b, int64_t nlevels, int use_graph);
int ps_batch_get_state(ps_batch *b, int index, double *dst, int level, int dst_on_device);
int ps_batch_synchronize(ps_batch *b);
int64_t ps_batch_launches(const ps_batch *b);
int ps_batch_units(const ps_batch *b);
const char *ps_batch_last_error(const ps_batch *b);

/*
 * Heat equation with a spatially varying diffusivity alpha(x, y) and its
 * adjoint.  No counterpart in the reference (its heat plugin has one scalar
 * ALPHA, pysweep/equations/heat.cu:8); the per-cell update keeps the plugin's
 * operation order with courant = alpha*dt/dx/dx per cell.  All pointers are
 * device pointers of nx*ny doubles; ny must be a multiple of 64.
 *
 * ps_heatvar_forward: u_T after nsteps steps from u0.  Writes the courant
 * field to d_courant, uses d_work as scratch, and (if d_checkpoints != NULL)
 * stores u every `every` steps: checkpoint k = u_{k*every}, k = 0 ..
 * ceil(nsteps/every)-1.
 *
 * ps_heatvar_adjoint: for J(u_T) with d_lamT = dJ/du_T, writes dJ/du0 to
 * d_lam0 and dJ/dalpha to d_galpha, walking the checkpoint segments backward:
 * each segment's states are recomputed into d_states (every fields), then the
 * adjoint steps lambda_n = lambda_{n+1} + L(C .* lambda_{n+1}),
 * dJ/dC += lambda_{n+1} .* L u_n run backward through it.  d_lamwork is a
 * scratch field.  `err` receives a message on failure.
 *
 * ps_heatvar_courant: only the courant field, d_courant = d_alpha*dt/dx/dx
 * (the values ps_heatvar_forward writes), for the swept form of the same
 * solve (PS_EQ_HEATVAR / PS_EQ_HEATVAR_ADJ solvers).
 *
 * ps_heatvar_recompute: the recompute of one checkpoint segment for the
 * swept adjoint: from d_u0 (the segment's checkpoint) runs `length` steps and
 * stores the Laplacian of every old level k = 0 .. length-1 at
 * d_lap[k][nx][ny] (the field 1 that PS_EQ_HEATVAR_ADJ(MU) solvers read);
 * d_work holds two fields of scratch.  Two steps per launch, the fused
 * forward kernels' arithmetic, so the Laplacians equal those the
 * PS_EQ_HEATVAR solver stores.
 */
int ps_heatvar_courant(const double *d_alpha, double *d_courant, int nx, int ny, double dt,
                       double dx, void *stream, char *err, size_t errlen);
int ps_heatvar_recompute(const double *d_courant, const double *d_u0, double *d_lap, int length,
                         int nx, int ny, double *d_work, void *stream, char *err, size_t errlen);
int ps_heatvar_forward(const double *d_u0, const double *d_alpha, double *d_uT, int nx, int ny,
                       int64_t nsteps, double dt, double dx, double *d_courant, double *d_work,
                       double *d_checkpoints, int every, void *stream, char *err, size_t errlen);
int ps_heatvar_adjoint(const double *d_courant, const double *d_checkpoints, int every,
                       const double *d_lamT, double *d_lam0, double *d_galpha, int nx, int ny,
                       int64_t nsteps, double dt, double dx, double *d_states, double *d_lamwork,
                       void *stream, char *err, size_t errlen);

/* Library version string. */
const char *ps_version(void);

#ifdef __cplusplus
}
#endif

#endif /* PYSWEEP_B200_H */
