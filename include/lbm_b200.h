/*
 * lbm_b200.h -- C ABI of the B200 time step of the D2Q9 MRT lattice-Boltzmann
 * flapping-airfoil solver (immersed boundary, implicit velocity correction).
 *
 * Every entry point replaces one Fortran subroutine (or one block of the
 * driver loop) of the reference R-IFFERY/Fortran_loadFile_mitiwing; the
 * citation next to each declaration names it (file:line in that project).
 *
 * Conventions
 *   - Every function returns an int status (LBM_OK == 0). No exception or
 *     longjmp crosses this boundary. lbm_last_error() gives the message of the
 *     last failing call on a handle.
 *   - Host arrays are Fortran order, x fastest, 1-based node (i,j) at
 *     index (i-1) + (j-1)*nx; populations (nx,ny,9) add (k-1)*nx*ny. Motion
 *     tables are (rows, cols) column-major, exactly as the Fortran driver
 *     holds motion_table(count, motion_column_count).
 *   - A handle owns all of its device memory and one CUDA stream. Host
 *     pointers are borrowed for the duration of a call only. Calls on one
 *     handle must be serialised by the caller; different handles may be
 *     driven from different host threads.
 *   - Device pointers never cross this ABI, except the velocity fields given
 *     to lbm_residual_device.
 */
#ifndef LBM_B200_H
#define LBM_B200_H

#include <stdint.h>

#if defined(__GNUC__)
#define LBM_API __attribute__((visibility("default")))
#else
#define LBM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define LBM_ABI_VERSION 1

/* status codes */
#define LBM_OK               0
#define LBM_DONE             1   /* time passed motion_end_time (main.f90:352-353) */
#define LBM_ERR_ARG         -1   /* bad argument / size */
#define LBM_ERR_CUDA        -2   /* CUDA runtime error, or no usable device */
#define LBM_ERR_STATE       -3   /* call out of order (e.g. step before init) */
#define LBM_ERR_IO          -4   /* file missing or malformed (mode.f90:82-135, airfoil.f90:224-234) */
#define LBM_ERR_SOLVER      -5   /* immersed-boundary system not positive definite / singular */
#define LBM_ERR_NONFINITE   -6   /* NaN/Inf seen in forces, in the flow at the markers or in the mass check */
#define LBM_ERR_RANGE       -7   /* a marker's support box reaches the three outermost node layers */
#define LBM_ERR_SIZE        -8   /* size beyond a fixed maximum (lbm_residual_device) */
#define LBM_ERR_INDEX       -9   /* a kernel found an index read from device memory out of range and
                                    skipped that access; the message names the kernel. Not expected:
                                    it means device state was overwritten (report it) */

/* storage precision of the populations (all collision arithmetic is FP32,
 * or FP64 for LBM_PREC_FP64; immersed-boundary solve and force sums are FP64) */
#define LBM_PREC_FP32  0
#define LBM_PREC_FP64  1
#define LBM_PREC_FP16  2
#define LBM_PREC_BF16  3

/* flags: solve the marker system with the dense Cholesky even when it is
 * banded (the path the solver otherwise takes only for couplings that reach
 * past the neighbouring 16-marker block); for verification */
#define LBM_FLAG_DENSE_SOLVE 1

/* discrete delta kernel (boundary_condition.f90:1530, 1563-1600) */
#define LBM_DELTA_PESKIN4  0   /* smooth=0: 4-point Peskin, support |r|<2   */
#define LBM_DELTA_SMOOTH   1   /* smooth=1: smoothed kernel, support |r|<=2.5 */

/* Run parameters. In the reference these are compile-time PARAMETERs of
 * module com_date (main.f90:4-137) and values set by ini_mesh
 * (ini_mesh.f90:15-67); here they are runtime values. */
typedef struct lbm_params {
    int32_t nx, ny;            /* mesh%Nx, mesh%Ny (ini_mesh.f90:22-23) */
    int32_t wing_count;        /* wing_count (main.f90:18) */
    int32_t points_per_wing;   /* boundary_points_per_wing (main.f90:21); closed contour */
    int32_t delta_kernel;      /* LBM_DELTA_*; the reference hard-codes smooth=1 */
    int32_t precision;         /* LBM_PREC_* */
    int32_t flags;             /* LBM_FLAG_* bits, else 0 */
    int32_t reserved;
    double scale;              /* mesh%scale: lattice spacing in chords (1/chord_lu) */
    double ox, oy;             /* mesh%ox, mesh%oy: physical position of node (1,1) */
    double uu;                 /* UU: lattice free-stream speed (main.f90:12) */
    double re;                 /* Re (main.f90:84); nu = uu/scale/re, tau = 3 nu + 0.5 */
    double s[9];               /* MRT rates mesh%s (ini_mesh.f90:59-67);
                                  s[7] or s[8] <= 0 means 1/tau_f */
    double xc, yc;             /* body reference point xc, yc (main.f90:85) */
    double xp, yp;             /* pivot xp, yp (main.f90:86) */
    double mesh_max_scale;     /* mesh_max_scale (main.f90:32), only scales movenum */
} lbm_params;

typedef struct lbm_handle lbm_t;

/* ---- set-up ------------------------------------------------------------ */

/* Fills p with the reference's own PARAMETER values (main.f90:7-137,
 * ini_mesh.f90:15-67): 4001x2001, scale 0.01, UU 0.01, Re 500, two wings of
 * 205 points, s=(0,1.1,1.05,0,1.2,0,1.2,1/tau,1/tau), smooth=1, FP32 storage. */
LBM_API int lbm_default_params(lbm_params *p);

/* ini_mesh (ini_mesh.f90:1-81): validates the parameters and allocates the
 * device state (two population buffers, IB scratch, step table). The device
 * memory comes from a stream-ordered pool that the library keeps per device
 * for the life of the process: memory a destroyed handle returned is reused
 * by the next handles without mapping it again. */
LBM_API int lbm_create(const lbm_params *p, lbm_t **out);

/* frees everything the handle owns (the reference frees nothing); its
 * device memory goes back to the library's pool (no device-wide
 * synchronisation) */
LBM_API int lbm_destroy(lbm_t *h);

/* read_boundary (airfoil.f90:207-242) for one wing from memory: npts
 * (= points_per_wing) points of a closed contour in chords, body frame.
 * Computes arc_l = |segment| / scale and applies the (xc-xp, yc-yp) shift
 * (airfoil.f90:235-241). wing is 1-based. */
LBM_API int lbm_set_boundary(lbm_t *h, int wing, const double *x, const double *y, int npts);

/* read_boundary from files: boundary.dat for wing 1 and boundary<w-1>.dat for
 * wing w (airfoil.f90:191-205), format (2f14.8), in directory dir ("" = cwd). */
LBM_API int lbm_read_boundary(lbm_t *h, const char *dir);

/* load_motion_table + build_motion_step_table(scale*UU) (mode.f90:68-142,
 * 245-269) from memory: table is (rows, cols) column-major with
 * cols = 1 + 9*wing_count (time, then per wing angle, omega, omgac, sa, sau,
 * saac, sb, sbv, sbac). Rejects an empty table and a decreasing time column. */
LBM_API int lbm_set_motion_table(lbm_t *h, const double *table, int rows, int cols);

/* load_motion_table from a motion_params.dat file (mode.f90:68-142). */
LBM_API int lbm_load_motion_table(lbm_t *h, const char *path);

/* Host-only parsers behind lbm_read_boundary / lbm_load_motion_table; they
 * need no device. The boundary parser reads npts (2f14.8) records of one file
 * (airfoil.f90:229). The motion parser reads the non-blank rows of a
 * list-directed motion_params.dat (mode.f90:88-123) into table (column-major,
 * max_rows x cols); *rows receives the row count (also when table is NULL,
 * which only counts). */
LBM_API int lbm_parse_boundary_file(const char *path, int npts, double *x, double *y);
LBM_API int lbm_parse_motion_file(const char *path, int cols, double *table, int max_rows, int *rows);

/* init (solution.f90:1-72) plus the driver's state reset (main.f90:294-328):
 * rho=1, u=UU, v=0, f=f0=feq with single-precision lattice weights.
 * du, dv (nx*ny each, nullable) are added to u and v before feq is taken;
 * they carry a seeded initial perturbation, which the reference does not
 * have (zero arrays reproduce it exactly). */
LBM_API int lbm_init(lbm_t *h, const double *du, const double *dv);

/* ---- the time step ---------------------------------------------------- */

/* One pass of the driver loop body (main.f90:352-359): time=(n-1)*scale*UU,
 * stop if time > motion_end_time+1e-12 (returns LBM_DONE), else
 * evolution (solution.f90:269-410): mode, move_boundary, streaming,
 * physical_variables, immersed_boundary_Wu, colission, force normalisation,
 * boundary_condition1. force_row (nullable, lbm_force_row_length doubles)
 * receives the force.dat row of this step (solution.f90:349-377). */
LBM_API int lbm_step(lbm_t *h, double *force_row);

/* nsteps passes of lbm_step, enqueued back to back on the device with no host
 * synchronisation in between (the main.f90:351-418 loop without output).
 * force_rows (nullable) receives nsteps rows, row-major, row length
 * lbm_force_row_length. *done_steps (nullable) = steps actually run; the run
 * stops early with LBM_DONE at motion_end_time. */
LBM_API int lbm_run(lbm_t *h, int nsteps, double *force_rows, int *done_steps);

/* length of one force.dat row: 1 + 3*wing_count + 3 + 9*wing_count
 * (solution.f90:350-375) */
LBM_API int lbm_force_row_length(const lbm_t *h);

/* ---- observation / checkpoint ---------------------------------------- */

/* the !$acc update host of rho, u, v (main.f90:408) as FP64 (nx,ny) arrays,
 * values after the boundary condition of the last step. Any pointer may be
 * NULL. */
LBM_API int lbm_get_fields(lbm_t *h, double *rho, double *u, double *v);

/* populations f(nx,ny,9) as FP64, after the last step (mesh%f). */
LBM_API int lbm_get_populations(lbm_t *h, double *f);

/* restores f(nx,ny,9) (readflowfield, solution.f90:1709-1839, the f part);
 * the edge f0 copies are kept from lbm_init (lbm_read_flow_field restores
 * them from a restart file). */
LBM_API int lbm_set_populations(lbm_t *h, const double *f);

/* erranalysis (solution.f90:74-127): ||u-u0|| / (||u|| + 1e-30) over the
 * interior, u from the last step and u0 from the state before it (the
 * initial field after one step). Needs one step run since init (else
 * LBM_ERR_STATE). */
LBM_API int lbm_residual(lbm_t *h, double *err);

/* Global mass sum_ij sum_k f_k of the populations after the last step,
 * summed on the device in FP64 in a fixed order (the same value on every
 * call for the same state). lbm_run also checks it at every copy of force
 * rows (every 2048 steps and at the end of the call), lbm_step on every
 * 2048th step and lbm_batch_run at the end of the call for each case; a
 * non-finite mass ends the run with LBM_ERR_NONFINITE. The reference has no
 * mass check; its lattice-wide reduction is erranalysis
 * (solution.f90:102-109). Returns LBM_ERR_NONFINITE (with *mass set) if the
 * mass is not finite. */
LBM_API int lbm_mass(lbm_t *h, double *mass);

/* immersed-boundary diagnostics of the last step: marker midpoints xb2,yb2
 * (airfoil.f90:267-270; n = wing_count*(points_per_wing-1) each), the
 * relative residual ||B y - rhs|| / ||rhs|| of the marker system solve, and
 * the half-bandwidth of B in the marker order the solver used (above 16 the
 * banded solver hands over to a dense Cholesky). Every pointer is nullable. */
LBM_API int lbm_get_markers(lbm_t *h, double *xb2, double *yb2, double *solve_residual, int *half_bandwidth);

/* Device timing of the step loop, the CUDA-event analogue of the driver's
 * per-phase cpu_time totals (main.f90:355-369, 420-433). With timing on,
 * enable = LBM_TIMING_KERNELS (or any other non-zero value but
 * LBM_TIMING_SPAN): lbm_step/lbm_run record CUDA events on the handle's
 * streams around the immersed-boundary kernels and around the lattice kernel
 * of every step. enable = LBM_TIMING_SPAN: only at the start and the end of
 * each run of up to 2048 steps, so that the steps are timed without the
 * per-step events in their streams (the kernel totals stay 0). 0: off.
 * lbm_get_timing returns, since the last lbm_set_timing, the summed device
 * milliseconds of the whole steps, of the immersed-boundary kernels and of
 * the lattice kernel, and the number of steps timed (any pointer nullable). */
#define LBM_TIMING_KERNELS 1
#define LBM_TIMING_SPAN 2
LBM_API int lbm_set_timing(lbm_t *h, int enable);
LBM_API int lbm_get_timing(lbm_t *h, double *step_ms, double *ib_ms, double *lattice_ms, int *steps);

/* Residual of erranalysis (solution.f90:74-122) on velocity fields held in
 * the CALLER's device memory, for drivers that keep u, v on the GPU
 * themselves (OpenACC or CUDA Fortran arrays, as the reference's own
 * erranalysis uses) and cannot let the library allocate: their arrays may
 * fill the device's memory, and an allocation or free per call would
 * synchronise the device. This entry point has no counterpart in the
 * reference. It needs no handle and allocates nothing: its scratch is one
 * fixed array in device memory per device, sized for at most
 * LBM_RESIDUAL_MAX_ROWS interior rows (ny - 2); a larger ny returns
 * LBM_ERR_SIZE and launches nothing.
 *   u, v, u0, v0: device arrays of nx*ny values (x fastest), FP64 or FP32
 *     as `precision` says (LBM_PREC_FP64 / LBM_PREC_FP32), on the current
 *     device; interior nodes only enter the sums, as in the reference.
 *   stream: a cudaStream_t, or NULL for the legacy default stream; the call
 *     copies the result to host memory, so it waits for that stream, and
 *     writes *err = ||u - u0|| / (||u|| + 1e-30).
 * The first call in each CUDA context (the device's primary context, or a
 * context the caller created and made current) looks up the scratch's
 * address in that context; make that first call before any stream capture.
 * Calls whose work overlaps on the GPU (other streams, other host threads on
 * the same device) share the scratch and race: serialise them. */
#define LBM_RESIDUAL_MAX_ROWS 16384
LBM_API int lbm_residual_device(const void *u, const void *v, const void *u0, const void *v0,
                                int nx, int ny, int precision, void *stream, double *err);

/* number of CUDA kernels this handle has launched since lbm_create (all
 * entry points: steps, population transfers, residuals). No counterpart in
 * the reference, which has no device code. */
LBM_API int lbm_get_launch_count(const lbm_t *h, long long *count);

/* current step counter n of the driver loop (1 before the first step). */
LBM_API int lbm_step_index(const lbm_t *h);

/* device memory the handle holds now, in bytes: lattice buffers and fields
 * from lbm_create, immersed-boundary scratch from the first step (FP64
 * staging for population transfers is made and released within each call).
 * Serving loops admit cases against an HBM budget with it. No counterpart
 * in the reference (one case per process there). */
LBM_API int lbm_device_bytes(const lbm_t *h, long long *bytes);

/* message of the last failing call on h ("" if none); h may be NULL for
 * errors of lbm_create. The string stays valid until the next call on h. */
LBM_API const char *lbm_last_error(const lbm_t *h);

/* Whether this library's kernels run on the current device:
 * *binary_version = the architecture they were compiled for (100 for
 * sm_100a, as cudaFuncAttributes::binaryVersion gives it) and *sm_count =
 * the device's multiprocessors (both nullable). LBM_ERR_CUDA when there is no
 * device or the device cannot load them. The reference picks its GPU target
 * at build time (nvfortran -gpu, Makefile:1-16) and has no such check. */
LBM_API int lbm_device_check(int *binary_version, int *sm_count);

/* The status code and message (into message[capacity], nullable) that a
 * device status word of the kernels turns into: the translation lbm_step /
 * lbm_run apply after each run of steps. Host only; needs no device. The
 * reference has no device status: its cuSOLVER status is ignored and bad
 * input stops the program (stop 1). */
LBM_API int lbm_describe_status(unsigned int status, char *message, int capacity);

/* ---- output and restart files -------------------------------------------
 * lbm_write_tecplot: the reference's output (solution.f90:129-238) for the
 *   state after the last step: Tecplot ASCII with the field zone sampled
 *   every stride_x-th / stride_y-th node from node 1 (the reference uses 2
 *   and 2; X, Y, U/UU, V/UU, pressure rho/3, vorticity dv/dx - du/dy with its
 *   one-sided differences on the edges, body and dvordt, written as 0: the
 *   live reference zeroes body after body_point, solution.f90:69, and never
 *   calls vor_mom_rate, main.f90:391), format (25e16.8), then the airfoil
 *   zone: contour points of the last step and one centre node per wing in
 *   (8f14.8), triangles in (3I5.3). `cycle` is the reference's n (file
 *   F<n>.dat; SOLUTIONTIME = n UU mesh_max_scale). Header lines are
 *   list-directed in spirit (values and order), not in one compiler's
 *   spacing.
 * lbm_write_tecplot_fields: the same file from host arrays (nx,ny) in
 *   Fortran order, without a handle (xb1, yb1: wing_count*points_per_wing
 *   contour points, nullable when wing_count = 0).
 * lbm_save_checkpoint / lbm_load_checkpoint: saveflowfield / readflowfield
 *   (solution.f90:1604-1839) as a two-file scheme: `path` and its copy (name
 *   with "_copy" before the extension, as saved_flow_feild_copy.dat), both
 *   written; the loader reads `path` and falls back to the copy when it is
 *   missing, short, from another grid or storage precision, or fails its
 *   checksum. The content is this library's own state (populations in
 *   storage precision, boundary reference values and the FP64 edge f0 they
 *   come from, both field slots, step counters), so a restart continues bit
 *   for bit; it is not the byte layout
 *   of the reference's form='binary' file. Load after lbm_init of a handle
 *   with the same parameters, boundary and motion table. */
LBM_API int lbm_write_tecplot(lbm_t *h, const char *path, int cycle, int stride_x, int stride_y);

/* output_gforce (solution.f90:240-267): the file g<n>.dat (n = cycle) with
 * the Eulerian force density gforce(Nx,Ny,2), host arrays in Fortran order
 * (x fastest; each nullable: zeros). The header line is written as (a), the
 * zone line list-directed in spirit; then one line of (25e25.17) per
 * position of the reference's loop as written, i = 1..Ny outer, j = 1..Nx
 * inner: ox+(i-1)scale, oy+(j-1)scale, gforce(i,j,1), gforce(i,j,2), with 0
 * for positions outside the array (j > Ny, reached when Nx > Ny). On the
 * live path gforce is 0 everywhere: move_boundary zeroes it at the support
 * nodes (airfoil.f90:280-281) and no routine of the live step writes it;
 * the live driver never calls output_gforce. */
LBM_API int lbm_write_gforce(const char *path, int cycle, int nx, int ny, double ox, double oy, double scale,
                             const double *gforce_x, const double *gforce_y);
LBM_API int lbm_write_tecplot_fields(const char *path, int nx, int ny, double ox, double oy, double scale, double uu,
                                     double solution_time, int stride_x, int stride_y, const double *rho,
                                     const double *u, const double *v, int wing_count, int points_per_wing,
                                     const double *xb1, const double *yb1);
LBM_API int lbm_save_checkpoint(lbm_t *h, const char *path);
LBM_API int lbm_load_checkpoint(lbm_t *h, const char *path);

/* ---- restart files in the reference's byte layout -----------------------
 * saveflowfield / readflowfield (solution.f90:1604-1839) as the reference
 * writes them: nvfortran form='binary' (no record markers, native byte
 * order): int32 cycle1, int32 wing_count, 11 x wing_count float64 body-state
 * arrays (body_rel_a, _a_prev, _v, _v_prev, _s, _s_prev, _pos, _theta_prev,
 * _theta, _temp_theta_prev, _temp_theta), int32 movenum; per node (j outer,
 * i inner) float64 u, v, f(1:9); then for j = 2..Ny-1 leftf2, f0(1,j),
 * rightf2, f0(Nx,j), and for i = 1..Nx upf2, f0(i,Ny), downf2, f0(i,1), 9
 * float64 each. A file written by the reference restarts this library and the
 * other way round. A restart continues bit for bit in FP32, FP16 and BF16
 * storage; FP64 storage keeps f - w, which the file's f holds only to f's
 * last bit, so an FP64 restart continues within rounding (about 1e-14 in f).
 * lbm_save_flow_field: the state after the last step into `path` and its copy
 *   (saved_flow_feild.dat and saved_flow_feild_copy.dat); cycle1 = the last
 *   step's number (lbm_step_index - 1); u, v of the last step (the step must
 *   have kept its fields, as for lbm_get_fields); leftf2 .. downf2 written as
 *   the edge f0 (both are the initial edge populations on the one-mesh path).
 *   body_state (11*wing_count, nullable = zeros) and movenum are the driver's
 *   rigid-body values, zero for prescribed motion.
 * lbm_read_flow_field: after lbm_init of the same case, reads `path`, or its
 *   copy when `path` is missing, short or of another size (LBM_ERR_IO when
 *   neither reads); a wing count other than the case's is LBM_ERR_STATE
 *   without trying the copy (the reference stops). Sets the populations, the
 *   boundary values from the file's edge f0, the fields (u, v from the file,
 *   density 1 as after init: the file has none) and the step counter (the
 *   next step is cycle1 + 1, main.f90:321-323). Returns cycle1, the body
 *   state and movenum (nullable); a file with non-zero body state or movenum
 *   (free flight, which this library does not model) is LBM_ERR_STATE and
 *   leaves the handle unchanged.
 * lbm_write_flow_field_file / lbm_read_flow_field_file: one file from / into
 *   host arrays, no handle and no device: u, v (nx,ny) and f (nx,ny,9) in
 *   Fortran order, edge_f0 = 9 float64 per node for the left column
 *   (j = 1..Ny), the right column, the bottom row (i = 1..Nx) and the top
 *   row. The reader returns LBM_ERR_IO (missing, short, other size) or
 *   LBM_ERR_STATE (other wing count). */
LBM_API int lbm_save_flow_field(lbm_t *h, const char *path, const double *body_state, int movenum);
LBM_API int lbm_read_flow_field(lbm_t *h, const char *path, int *cycle, double *body_state, int *movenum);
LBM_API int lbm_write_flow_field_file(const char *path, int nx, int ny, int cycle, int wing_count,
                                      const double *body_state, int movenum, const double *u, const double *v,
                                      const double *f, const double *edge_f0);
LBM_API int lbm_read_flow_field_file(const char *path, int nx, int ny, int wing_count, int *cycle,
                                     double *body_state, int *movenum, double *u, double *v, double *f,
                                     double *edge_f0);

/* ---- batches: several cases stepped together on one GPU ----------------
 * The reference runs one case per process (main.f90); flapping-wing studies
 * are sweeps of many cases. A batch steps initialised handles of different
 * grid sizes and kinematics with one launch per kernel for all of them: one
 * lattice launch driven by a case table, and each immersed-boundary stage as
 * one launch over the cases. Cases may be at different steps, and may join
 * and leave between runs (the serving loop of the Python layer does so).
 * Each case's results are bit-for-bit those of running it alone (lbm_run).
 * The batch does not own the handles; between runs a case may also be
 * stepped alone.
 *   lbm_batch_create: cases (count >= 0) must be initialised, share storage
 *     precision, factorization batch and device, and have markers.
 *   lbm_batch_add / lbm_batch_remove: a case joins (same conditions) or
 *     leaves the batch; the order of the remaining cases is kept.
 *   lbm_batch_count: cases in the batch.
 *   lbm_batch_case_status: status of case c (batch order) in the last
 *     lbm_batch_run: LBM_OK or the error code its checks raised, with the
 *     message in lbm_last_error of that case. A run stops at the first check
 *     that finds a failed case (a diverged flow, say); the rows and steps of
 *     every case up to that check are delivered, and the other cases stay
 *     valid and may go on in the next run once the failed one is removed.
 *   lbm_batch_run: runs up to nsteps steps of every case; a case stops when
 *     its motion table ends (done_steps[c], nullable; LBM_DONE when any case
 *     ran fewer than nsteps). force_rows[c] (nullable, or an array of
 *     nullable pointers) receives case c's rows as lbm_run would. Fields are
 *     kept for the last two steps of the call and of each case that ends.
 *   lbm_batch_set_rows: rows per CTA of the lattice kernel for the batch
 *     (0: the cases' own); the batch autotuner of the Python layer sets it.
 *   lbm_batch_set_occupancy: at most ctas_per_sm (1..8) CTAs of the batch's
 *     lattice kernel on an SM, by asking each CTA for that share of the
 *     SM's shared memory (0, the default: as many as the registers allow,
 *     4 for 2- and 4-byte storage); the autotuner sets it beside the rows.
 *   lbm_batch_get_timing: device milliseconds of the last lbm_batch_run's
 *     steps (CUDA events on the batch's streams, from before the first
 *     step's launches to the end of the last step) and the number of steps
 *     it ran; 0 after a run that failed.
 *   lbm_batch_set_graphs: 1 (the default; environment LBM_BATCH_GRAPHS=0
 *     turns it off at creation) runs steady steps as CUDA graphs of 16
 *     steps: wherever the next 16 steps keep the same active cases and
 *     write no fields (not the first step of a run, nor the last two of the
 *     call or of a case), the batch replays an instantiated graph of those
 *     steps' launches, captured the first time a segment of that structure
 *     occurs and kept (up to 8 per batch; adding or removing a case drops
 *     them), after rewriting the host copy of the argument buffer the
 *     graph's first node uploads. 0 issues every step's launches from the
 *     host. The results are the same bit for bit.
 *   lbm_batch_graph_stats: steps run as graph segments, graph launches and
 *     graphs instantiated over the batch's life (each nullable). */
typedef struct lbm_batch lbm_batch_t;
LBM_API int lbm_batch_create(lbm_t *const *cases, int count, lbm_batch_t **out);
LBM_API int lbm_batch_destroy(lbm_batch_t *b);
LBM_API int lbm_batch_add(lbm_batch_t *b, lbm_t *h);
LBM_API int lbm_batch_remove(lbm_batch_t *b, lbm_t *h);
LBM_API int lbm_batch_count(const lbm_batch_t *b);
LBM_API int lbm_batch_case_status(const lbm_batch_t *b, int c);
LBM_API int lbm_batch_set_rows(lbm_batch_t *b, int rows_per_cta);
LBM_API int lbm_batch_set_occupancy(lbm_batch_t *b, int ctas_per_sm);
LBM_API int lbm_batch_set_graphs(lbm_batch_t *b, int enable);
LBM_API int lbm_batch_graph_stats(const lbm_batch_t *b, long long *graph_steps, long long *graph_launches,
                                  long long *graph_builds);
LBM_API int lbm_batch_get_timing(const lbm_batch_t *b, double *ms, int *steps);
LBM_API int lbm_batch_run(lbm_batch_t *b, int nsteps, double *const *force_rows, int *done_steps);
LBM_API const char *lbm_batch_last_error(const lbm_batch_t *b);

#ifdef __cplusplus
}
#endif

#endif /* LBM_B200_H */
