/* femorph_b200: B200-native explicit stabilised incompressible-flow step.
 *
 * C ABI of the library libfemorph_b200.so.  Plain structs of pointers and
 * sizes, 0-based int32 connectivity, FP64 coordinates and state.  The caller
 * owns every host buffer it passes; the library owns the device buffers.
 * Every function returns FM_OK (0) or an FM_ERR_* code; no C++ exception
 * crosses this boundary.  Handles are not thread-safe: one host thread per
 * batch at a time.
 *
 * The entry points replace these reference interfaces (desResLab/feMorph):
 *   femVMSExplicitFluidSolver::solve(femModel*)   src/femVMSExplicitFluidSolver.h:9-14,
 *                                                 src/femVMSExplicitFluidSolver.cpp:842-1334
 *   femSUPGExplicitFluidSolver::solve(femModel*)  src/femSUPGExplicitFluidSolver.h:9-14,
 *                                                 src/femSUPGExplicitFluidSolver.cpp:794-1735
 *   femModel public fields read by those solvers  src/femModel.h:24-108
 *   femModel::ReadFromFEMTextFile                 src/femModel.cpp:3719-4213
 *   femModel::ExportToVTKLegacy                   src/femModel.cpp:1294-1530
 * The femSolver adapter classes that keep the reference's
 * solve(femModel*) entry live in femorph_b200/adapter/.
 */
#ifndef FEMORPH_B200_H
#define FEMORPH_B200_H

#include <stdint.h>

#if defined(__GNUC__)
#define FM_API __attribute__((visibility("default")))
#else
#define FM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- return codes ---- */
enum {
  FM_OK = 0,
  FM_ERR_INVALID = 1,     /* bad argument, unsupported option or malformed input */
  FM_ERR_OOM = 2,         /* device or host allocation failed */
  FM_ERR_CUDA = 3,        /* a CUDA runtime call failed */
  FM_ERR_DIVERGED = 4,    /* NaN/Inf in the state, or max |u| above EXITCOND */
  FM_ERR_TIMEOUT = 5,     /* a bounded device-side wait gave up */
  FM_ERR_TABLE = 6,       /* time outside a NODEVEL table (femUtils.cpp:852-860) */
  FM_ERR_IO = 7,          /* file could not be read or written */
  FM_ERR_NODEVICE = 8     /* no usable sm_100 device */
};

enum { FM_TET4 = 4, FM_HEXA8 = 8 };
enum { FM_SOLVER_VMS = 0, FM_SOLVER_SUPG = 1 };
enum { FM_FP64 = 0, FM_MIXED = 1 };
/* FM_MIXED (VMS and SUPG): Gauss-point work in FP32, nodal accumulation,
 * history, lumped-mass division and state in FP64.  Elements whose aspect
 * ratio exceeds this limit keep their Jacobian inverse in FP64: tets by
 * h_max / (2 sqrt(6) r_in) (regular tet 1.0, Kuhn tet 1.7), hexa8 by longest
 * over shortest edge (cube 1.0). */
#define FM_MIXED_ASPECT_LIMIT 3.0
/* Size of the fixed device array behind fm_vms_solve_static (32 MiB). */
#define FM_STATIC_SCRATCH_BYTES (32u << 20)
/* NODEDOF global fixed dofs (femSUPGExplicitFluidSolver.cpp:1527-1561) */
enum { FM_FIX_NONE = 0, FM_FIX_X = 1, FM_FIX_Y = 2, FM_FIX_Z = 4 };

/* Mesh: femModel::nodeList / elementList (femModel.h:26-27). */
typedef struct fm_mesh {
  int32_t elem_type;      /* FM_TET4 or FM_HEXA8 (hexa8 only with SUPG) */
  int64_t n_nodes;
  int64_t n_elems;
  const double* coords;   /* n_nodes x 3 */
  const int32_t* conn;    /* n_elems x elem_type, 0-based */
} fm_mesh;

/* Boundary conditions exactly as the .dat rows define them
 * (femModel.cpp:3941-4005): NODEVEL rows in file order (grouped into per-node
 * time tables by femModel::postProcessNodeVelocities, femModel.cpp:4549-4576),
 * NODEDIRBC rows, NODEPRES rows. */
typedef struct fm_bc {
  int64_t n_vel_rows;
  const int32_t* vel_node;   /* node of each row */
  const double* vel_vals;    /* rows x 4: vx, vy, vz, time */
  const int32_t* vel_dir;    /* 0..6: X Y Z XY YZ XZ XYZ */
  int64_t n_dir;
  const int32_t* dir_node;
  const double* dir_vals;    /* n_dir x 3 */
  int64_t n_pres;
  const int32_t* pres_node;
  const double* pres_vals;
} fm_bc;

/* Solver parameters: femModel.h fields vmsProps, timeStep, totalSteps,
 * saveEvery, dual_step, tot_dual_steps, exOpts, glob_fixed_dofs,
 * exit_condition. */
typedef struct fm_params {
  int32_t solver;          /* FM_SOLVER_VMS or FM_SOLVER_SUPG */
  int32_t precision;       /* FM_FP64 or FM_MIXED */
  double props[5];         /* VMS: rho mu invEps c1 c2; SUPG: rho mu alpha cI - */
  double time_step;
  int32_t total_steps;     /* TIMESTEP: the reference runs total_steps-1 steps */
  int32_t save_every;
  double dual_step;        /* VMS DUALSTEP */
  int32_t tot_dual_steps;  /* VMS: dual iterations per step = tot_dual_steps+1 */
  int32_t ex_opts[6];      /* SUPG EXOPTS: euler, B-bar, K1, K2, K3, K4 */
  int32_t glob_fixed;      /* SUPG FM_FIX_* mask */
  double exit_condition;   /* SUPG EXITCOND (max |u|); <= 0 disables */
} fm_params;

/* Launch shape; zero fields take the built-in defaults (or the autotuned
 * values when fm_batch_autotune has run). */
typedef struct fm_tuning {
  int32_t tile_elems;      /* elements per tile (one CTA owns one tile)  */
  int32_t tile_nodes;      /* max distinct nodes per tile (shared memory) */
  int32_t threads;         /* threads per CTA */
  int32_t graph_steps;     /* time steps captured per CUDA graph (0: no graph) */
  int32_t ctas_per_sm;     /* VMS register budget: the tile kernel variant compiled for at least this
                            * many resident CTAs an SM (registers a thread <= 65536 / (threads x
                            * ctas_per_sm)); 0 takes the default.  128 threads: FP64 3 (default) or 4,
                            * mixed 4 (default) or 5; 256 threads: FP64 1 (default) or 2, mixed 2.
                            * SUPG ignores it. */
  int32_t reserved[3];
} fm_tuning;

/* Pool capacities of a batch created empty (fm_batch_create_empty).  The
 * batch's problems all share solver, element type and precision. */
typedef struct fm_capacity {
  int32_t solver;          /* FM_SOLVER_* */
  int32_t elem_type;       /* FM_TET4 / FM_HEXA8 */
  int32_t precision;       /* FM_FP64 / FM_MIXED */
  int32_t max_problems;    /* resident problems at the same time */
  int64_t max_elems;       /* resident elements, all problems together */
  int64_t max_nodes;       /* resident nodes, all problems together */
  int64_t max_table_rows;  /* NODEVEL table rows, all problems (0: max_nodes) */
  int64_t reserved[4];
} fm_capacity;

typedef struct fm_problem fm_problem;
typedef struct fm_batch fm_batch;

FM_API const char* fm_strerror(int code);
FM_API const char* fm_last_error_message(void);
FM_API int fm_version(void);

/* Host-side problem description.  init_state (n_nodes x 4: u v w p, before
 * BCs) may be NULL for a zero start.  The library copies what it needs. */
FM_API int fm_problem_create(const fm_mesh* mesh, const fm_bc* bc, const fm_params* params,
                      const double* init_state, fm_problem** out);
FM_API int fm_problem_destroy(fm_problem* p);

/* Reads a reference .dat keyword file (femModel::ReadFromFEMTextFile,
 * femModel.cpp:3719-4213; NODE, ELEMENT TET4|HEXA8, NODEVEL, NODEDIRBC,
 * NODEPRES, NODEDOF, TIMESTEP, DUALSTEP, VMSPROPS, EXOPTS, EXITCOND; other
 * keywords are ignored).  solver and precision are taken from the optional
 * keywords "SOLVER VMS|SUPG" and "PRECISION FP64|MIXED", else from the
 * arguments. */
FM_API int fm_problem_read_dat(const char* path, int32_t solver, int32_t precision, fm_problem** out);

/* Sizes of a problem (any pointer may be NULL). */
FM_API int fm_problem_info(const fm_problem* p, int64_t* n_nodes, int64_t* n_elems, int32_t* elem_type,
                    int32_t* solver, int64_t* steps_done);

/* Packs problems into one device-resident batch (one launch per time step
 * for all of them).  device: CUDA ordinal.  The problems must outlive the
 * batch. */
FM_API int fm_batch_create(fm_problem* const* problems, int32_t n, const fm_tuning* tuning, int32_t device,
                    fm_batch** out);
FM_API int fm_batch_destroy(fm_batch* b);

/* Continuous batching.  fm_batch_create_empty allocates device pools of the
 * given capacities once; fm_batch_add places a problem into free ranges of
 * them (its state starts at the time-0 BCs, as in fm_batch_create) and
 * returns FM_ERR_OOM when some pool has no room, leaving the batch as it was;
 * fm_batch_remove frees a problem's ranges (its results are lost: read them
 * first).  Both wait for the batch's stream.  A problem's stepping and
 * results do not depend on which other problems share its batch.
 * fm_problem_prepare builds the problem's tile layout ahead of
 * fm_batch_add/fm_batch_create (host only; different problems may be
 * prepared on different threads).  None of these has a counterpart in the
 * reference, which solves one model per process (femSolver::solve). */
FM_API int fm_batch_create_empty(const fm_capacity* cap, const fm_tuning* tuning, int32_t device, fm_batch** out);
FM_API int fm_batch_add(fm_batch* b, fm_problem* p);
FM_API int fm_batch_remove(fm_batch* b, fm_problem* p);
FM_API int fm_problem_prepare(fm_problem* p, const fm_tuning* tuning);
/* Builds (or reuses) the problem's tile layout for these tile sizes and
 * checks the invariants the tile kernels rely on: local connectivity inside
 * each tile's node list, interior nodes touched by one tile only, no two
 * elements of a colour sharing a node, each (element, corner) once in its
 * node's incidence list in element order, one partial slot per (tile,
 * interface node) listed in tile order, every element and node once; for a
 * partition part (fm_problem_partition) also that shared nodes are interface
 * nodes carrying their exchange index.
 * FM_ERR_INVALID names the first broken one.  Host only.  No counterpart in
 * the reference (its element loop neither tiles nor colours). */
FM_API int fm_problem_check_layout(fm_problem* p, const fm_tuning* tuning);
/* Device bytes fm_batch_create_empty allocates for these capacities (HBM
 * budgeting). */
FM_API int fm_batch_capacity_bytes(const fm_capacity* cap, const fm_tuning* tuning, int64_t* bytes);

/* Resident problems, their elements and the largest free run of element
 * slots (admission control). */
FM_API int fm_batch_resident(fm_batch* b, int32_t* problems, int64_t* elems, int64_t* largest_free_elems);

/* VMS solve that allocates no device memory, for callers that cannot call
 * cudaMalloc: a process whose device memory another allocator already holds
 * (a framework's caching allocator), or a latency-bound path on which
 * cudaMalloc/cudaFree, which synchronise the whole device, are not
 * acceptable.  It has no counterpart in the reference.
 *
 * Runs nsteps time steps of problem p (VMS, tet4, FP64; fm_problem_prepare
 * must have built its tile layout) from its initial state with the same
 * kernels as fm_batch_step, and writes the final velocity (n_nodes x 3) and
 * pressure (n_nodes) to the host arrays u and pres (either may be NULL),
 * in the problem's node numbering.  All device data - the problem's copy
 * and the kernels' scratch - lives in one fixed array of
 * FM_STATIC_SCRATCH_BYTES per GPU, held from the time the library's device
 * code is loaded on that GPU (at the latest the first call) until the
 * process exits.  Problems that need more (above roughly 200,000
 * tetrahedra) are rejected with FM_ERR_INVALID.  The first call on a device
 * looks up the array's device address and sets the kernels' shared-memory
 * limit; make that first call before any stream capture on the device.
 * Every call shares the array: calls that overlap on the GPU (from
 * different host threads or streams) race and must be serialised by the
 * caller.  Each call clears what has to start at zero.  stream: a
 * cudaStream_t (NULL: the default stream); the call returns after the
 * stream has finished its work. */
FM_API int fm_vms_solve_static(fm_problem* p, int32_t nsteps, int32_t device, double* u, double* pres, void* stream);

/* Advances every problem of the batch by nsteps time steps (VMS: each with
 * tot_dual_steps+1 dual iterations) on the given cudaStream_t (NULL: the
 * batch's own stream).  Asynchronous; fm_batch_sync waits and reports the
 * first device-side error (FM_ERR_DIVERGED, FM_ERR_TABLE, FM_ERR_TIMEOUT). */
FM_API int fm_batch_step(fm_batch* b, int32_t nsteps, void* stream);
FM_API int fm_batch_sync(fm_batch* b);

/* Per-problem step targets for ragged batches: the i-th resident problem
 * (in the order of the fm_batch_create array; problems added later follow
 * in slot order) advances by nsteps[i] (0 = idle). */
FM_API int fm_batch_step_ragged(fm_batch* b, const int32_t* nsteps, void* stream);

/* Advances only the listed problems (each by its nsteps entry); the rest of
 * the batch idles. */
FM_API int fm_batch_step_problems(fm_batch* b, fm_problem* const* problems, const int32_t* nsteps, int32_t count,
                                  void* stream);

/* ---- one mesh split over several GPUs (partition parts) ----
 * No reference counterpart: the reference solves one mesh in one process
 * (femVMSExplicitFluidSolver::solve / femSUPGExplicitFluidSolver::solve loop
 * over all elements, src/femVMSExplicitFluidSolver.cpp:1098-1208,
 * src/femSUPGExplicitFluidSolver.cpp:1095-1514); these calls split exactly
 * that loop.  A part owns some elements; nodes touched by several parts
 * (and, for VMS, the problem's nodes 0..3, whose pressures every element
 * reads) form the partition's exchange list.  Each dual iteration (VMS) or
 * step (SUPG) has one exchange: the parts' partial sums at those nodes,
 * 4 doubles a node, are added across parts, and every part updates its own
 * copy from the same sum.  Masses and BCs are the whole mesh's. */

/* Default split: n_parts bands of equal element count along the Morton
 * order of the element centroids.  elem_part: n_elems entries, out. */
FM_API int fm_partition_elements(const fm_problem* full, int32_t n_parts, int32_t* elem_part);
/* The problem of one part (elem_part NULL: the default split).  Its nodes
 * are the ones its elements touch (plus nodes 0..3 for VMS) in global
 * order; fm_problem_get_state and the other per-problem calls work in that
 * local numbering.  full stays valid and unchanged. */
FM_API int fm_problem_partition(const fm_problem* full, const int32_t* elem_part, int32_t n_parts, int32_t part,
                                fm_problem** out);
/* part index, part count and exchange-list length (part -1: not a part). */
FM_API int fm_problem_part_info(const fm_problem* p, int32_t* part, int32_t* n_parts, int64_t* x_total);
/* Global node / element of each local one, and each local node's index in
 * the exchange list (-1: not shared).  NULL arguments are skipped. */
FM_API int fm_problem_part_map(const fm_problem* p, int32_t* node_global, int32_t* elem_global, int32_t* xidx);

/* A batch created from partition parts (fm_batch_create, parts of one
 * partition only) gives each part a slice of a packed exchange buffer:
 * send and recv hold count = parts_in_batch x x_total x 4 doubles.  When
 * the batch holds every part, fm_batch_step runs the exchange itself
 * (recv == send).  Otherwise the other parts run in other processes (every
 * process with the same number of parts in its batch) and each iteration
 * is driven as
 *   fm_batch_exchange_begin(b, stream);   tile kernel + partial sums -> send
 *   <recv = sum over processes of send, enqueued on stream,
 *    e.g. ncclAllReduce(send, recv, count, ncclDouble, ncclSum, comm, stream)>
 *   fm_batch_exchange_end(b, stream);     shared nodes updated from recv
 * with all three on one cudaStream_t (NULL means the batch's own stream,
 * not the legacy default stream).  fm_batch_iterations_per_step gives the
 * iterations of one time step (VMS: tot_dual_steps + 1, SUPG: 1). */
FM_API int fm_batch_exchange_buffers(fm_batch* b, double** send, double** recv, int64_t* count);
FM_API int fm_batch_exchange_begin(fm_batch* b, void* stream);
FM_API int fm_batch_exchange_end(fm_batch* b, void* stream);
FM_API int fm_batch_iterations_per_step(fm_batch* b, int32_t* per_step);
/* begin/end pairs may be captured in a CUDA graph together with the
 * caller's reduction (after one pair has run outside the capture); a captured
 * pair counts no iteration, so after replaying a graph of k pairs the caller
 * reports them here (steps done, per-problem iteration counts). */
FM_API int fm_batch_exchange_account(fm_batch* b, int32_t iterations);

/* Velocity extrema of a problem's current state, reduced on the device
 * (get_solution_extrema, femSUPGExplicitFluidSolver.cpp:604-655; SUPG
 * global fixed dofs masked): out[0..5] min/max of u, v, w, out[6] max |u|. */
FM_API int fm_problem_velocity_extrema(fm_problem* p, double* out);

/* SUPG log quantities of the state about to be stepped, reduced on the
 * device as the reference's element loop accumulates them
 * (femSUPGExplicitFluidSolver.cpp:1066-1091, 1180-1245, 1430-1459, printed at
 * :1594-1630): out[0..1] min/max tau_SUPG, out[2..3] min/max lambda at the
 * Gauss points, out[4..6] max viscous, advective and lambda CFL, out[7..8]
 * min/max E and out[9..10] min/max nu of the element-averaged lambda.  (The
 * reference never resets its lambda CFL maximum between steps; a caller that
 * prints its log keeps that running maximum.) */
FM_API int fm_problem_supg_log_stats(fm_problem* p, double* out);

/* VMS diagnostics: the reference's per-dual-iteration log line and its
 * res_v / res_p output (femVMSExplicitFluidSolver.cpp:699-711,
 * 774-793, 1202-1215; the centroid residuals are quarter-weighted nodal
 * residuals read right after each element's assembly, i.e. running sums in
 * the reference's element order, rebuilt on the device from the
 * iteration's element residuals).  fm_batch_set_diagnostics(b, 1) makes
 * every later dual iteration of the batch's VMS problems record them
 * (slower: no CUDA graphs, extra passes and a host read per iteration;
 * 0 turns it off and frees the buffers).  fm_problem_vms_log pops up to
 * max_rows queued rows, oldest first, 6 doubles each: step (0-based),
 * dual iteration (1-based), time, max centroid |res_u|, max |res_p|, CFL;
 * rows NULL only reports the queued count in n_rows.
 * fm_problem_vms_residuals copies the last recorded iteration's centroid
 * residuals (res_u n_elems x 3, res_p n_elems; either may be NULL). */
FM_API int fm_batch_set_diagnostics(fm_batch* b, int32_t enable);

/* Failure detection (femSUPGExplicitFluidSolver.cpp:1635-1643 is the
 * reference's only failure exit; it has no device waits).  The VMS tile
 * kernel's waits for each chunk's bulk copies are bounded: after `polls`
 * unsuccessful mbarrier polls (default 4,194,304) the CTA waits, again
 * bounded, for the copies it issued, leaves its nodes untouched and sets the
 * problem's status to FM_ERR_TIMEOUT, which fm_batch_sync reports.  A
 * problem whose status is not FM_OK stops there: the kernels skip it from
 * then on.  A small limit (0: give up at once) makes the timeout path run on
 * demand, which is how it is tested; 0 is not for production use.  Drops
 * the batch's captured CUDA graph (it holds the old limit). */
FM_API int fm_batch_set_wait_limit(fm_batch* b, uint32_t polls);

/* Self-check of the device arithmetic that stands in for CUDA's division,
 * rcbrt and sqrt in the element kernels (Newton-Raphson from the PTX
 * approximate FP32 instructions).  No reference counterpart: the reference
 * computes 1.0 / detJ, pow(6V, 1/3) and sqrt on the host
 * (femVMSExplicitFluidSolver.cpp:64, 75, 585).  For each x[i] writes
 * out[i*8 .. i*8+7] = rcp_nr(x), 1.0/x, rcbrt_nr(x), rcbrt(x), sqrt_nr(x),
 * sqrt(x), rcbrt_nr((float)x), rcbrtf((float)x), computed on device 0
 * (allocates; for tests). */
FM_API int fm_math_check(const double* x, int64_t n, double* out);
FM_API int fm_problem_vms_log(fm_problem* p, double* rows, int32_t max_rows, int32_t* n_rows);
FM_API int fm_problem_vms_residuals(fm_problem* p, double* res_u, double* res_p);

/* Device status of one problem of a batch (FM_OK, FM_ERR_DIVERGED,
 * FM_ERR_TABLE, FM_ERR_TIMEOUT); waits for the batch's stream. */
FM_API int fm_problem_status(fm_problem* p);

/* Copies a problem's current state to host memory, in the problem's own
 * node/element numbering.
 *   u: n_nodes x 3 velocity;
 *   p: VMS n_nodes nodal pressure, SUPG n_elems element pressure
 *      (compute_pressure, femSUPGExplicitFluidSolver.cpp:446-501);
 *   elem3: VMS n_elems x 3 centroid subgrid velocity (subgrid_u of the VTK
 *      output), SUPG n_elems x 2 (lambda, regime);
 *   sdus: VMS n_elems x 12 Gauss-point subscales [e][gp][c] (SUPG: unused).
 * Any pointer may be NULL. */
FM_API int fm_problem_get_state(fm_problem* p, double* u, double* pres, double* elem3, double* sdus);

/* Writes the problem's current state as legacy ASCII VTK in the layout of
 * femModel::ExportToVTKLegacy (femModel.cpp:1294-1530).  The three writers
 * export the state of a problem in a batch; a problem not yet placed (or
 * placed and removed without a step) exports the initial state given at
 * fm_problem_create (zeros without one, before the Dirichlet values that
 * placement applies) with zero element fields; one that left its batch
 * after stepping is refused (FM_ERR_INVALID). */
FM_API int fm_problem_write_vtk(fm_problem* p, const char* path);
/* The same sections in legacy BINARY VTK (big-endian float32 points, int32
 * cells, float64 data); no counterpart in the reference, which writes ASCII
 * only. */
FM_API int fm_problem_write_vtk_binary(fm_problem* p, const char* path);
/* The same sections as VTK XML UnstructuredGrid (.vtu) with raw appended
 * little-endian arrays (FP64 points and data, int32 connectivity); no
 * counterpart in the reference. */
FM_API int fm_problem_write_vtu(fm_problem* p, const char* path);

/* Checkpoint and restart (no counterpart in the reference, whose VTK output
 * keeps six digits and cannot restart a solve).  fm_problem_checkpoint
 * writes everything the next iteration reads of a problem in a batch, in
 * the problem's own node / element numbering: the state after and before
 * BCs, the element state (VMS subscales, FP64 or FP32 as the precision
 * keeps them; SUPG history and lambda / regime), the iteration and step
 * counters, time, status and the pressures of nodes 0..3 (little-endian,
 * a 160-byte header then columns; layout in fm_runtime.cu).
 * The file is written to path.tmp and renamed over path when complete, so
 * a failed write leaves an earlier checkpoint at path intact.
 * fm_problem_restore loads such a file into a problem of the same mesh,
 * parameters (properties, time and dual step, dual iterations, EXOPTS,
 * fixed dofs, exit condition), BC rows and tables, solver and precision
 * that sits in a batch (any batch, any slot); stepping
 * on continues the solve: bit for bit the uninterrupted one when the batch
 * has the same tile sizes and threads.  Either call waits for the batch's
 * stream; neither may run while an exchange is open.  FM_ERR_IO for a file
 * error, FM_ERR_INVALID for a file of another mesh or configuration. */
FM_API int fm_problem_checkpoint(fm_problem* p, const char* path);
FM_API int fm_problem_restore(fm_problem* p, const char* path);

/* Nodal lumped mass as the solver uses it, problem numbering: VMS n_nodes
 * (initial_assemble, femVMSExplicitFluidSolver.cpp:87-89), SUPG n_nodes x 3
 * (form_lumped_mass, femSUPGExplicitFluidSolver.cpp:507-598). */
FM_API int fm_problem_get_mass(fm_problem* p, double* mass);

/* Device time of the kernels launched by the last fm_batch_step: total
 * milliseconds and the number of kernel launches (CUDA events on the batch
 * stream; valid after fm_batch_sync). */
FM_API int fm_batch_last_timing(fm_batch* b, double* ms, int64_t* launches);

/* Advances the batch by nsteps like fm_batch_step, bracketing every kernel
 * launch with CUDA events on the batch stream, and returns the summed device
 * time of the element (tile) kernel in kernel_ms[0] and of the interface
 * kernel in kernel_ms[1], with their launch counts.  Synchronous. */
FM_API int fm_batch_profile(fm_batch* b, int32_t nsteps, double* kernel_ms, int64_t* launches);

/* Autotuner: times the tile/interface kernels of these problems (as one
 * batch, `steps` steps per candidate, per-kernel CUDA events) over the
 * candidate launch shapes (tile elements x threads per CTA) and writes the
 * fastest to *best.  With cache_path non-NULL the result is looked up first
 * and stored afterwards, keyed by GPU name, solver, element type, precision
 * and the batch's element count (rounded to a power of two).  The problems
 * must not be in a batch; their host data is not modified. */
FM_API int fm_autotune(fm_problem* const* problems, int32_t n, int32_t device, int32_t steps, const char* cache_path,
                       fm_tuning* best);

/* Bytes of device memory a batch of these problems needs (admission). */
FM_API int fm_batch_estimate_bytes(fm_problem* const* problems, int32_t n, const fm_tuning* tuning, int64_t* bytes);

/* Layout statistics: tiles, interface nodes, max colours per tile. */
FM_API int fm_batch_layout(fm_batch* b, int64_t* n_tiles, int64_t* n_iface_nodes, int32_t* max_colors,
                    int64_t* n_slots);

/* ---- Poisson solver (femPoissonSolver::solve, femSolver.cpp:409-654) ----
 * The implicit neighbour of the explicit path: the same tet4 / hexa8
 * kinematics (irSecondOrder Gauss points, femElement.cpp:272-354) assemble
 *   K[a][b] = sum_e sum_g (sum_d diff_e[d] dN_a,d dN_b,d) detJ w_g
 * (femElement::formPoissonMatrix, femElement.cpp:903-944) and
 *   f[a] = sum_sources sum_g N_a source detJ w_g
 * (femElement::formPoissonSource, femElement.cpp:949-981), plus face Neumann
 * values spread evenly over the face's nodes (femSolver.cpp:546-562); the
 * Dirichlet rows become identity rows with the value on the right-hand side
 * (femTrilinosMatrix::applyBlockDirichelet, femTrilinosVector.cpp:109-119).
 * The reference then solves with Trilinos (its other builds stop: "Solver not
 * available", femSolver.cpp:590-600); here the system is solved on the GPU by
 * conjugate gradients with a Jacobi preconditioner on the assembled matrix
 * (the Dirichlet columns moved to the right-hand side, which keeps it
 * symmetric and leaves the solution unchanged).  Results: the nodal solution
 * ("PoissonResult"; its average subtracted for FM_POISSON_PPE,
 * femSolver.cpp:604-612) and, for FM_POISSON_DISTANCE, the element wall
 * distance of femPoissonSolver::evalDistanceFromPoissonSolution
 * (femSolver.cpp:366-403). */
enum { FM_POISSON_CLASSIC = 0, FM_POISSON_PPE = 1, FM_POISSON_DISTANCE = 2 };

/* femModel fields read by femPoissonSolver::solve (femModel.h): the mesh,
 * elDiffusivity (one row a element, in ELDIFF row order, femModel.cpp:
 * 3909-3925), sourceElement / sourceValues (ELSOURCE, femModel.cpp:
 * 3999-4011), neumannBCFaceNodes / neumannBCValues (FACENEUMANN,
 * femModel.cpp:4185-4200, face node lists in CSR form), diricheletBCNode and
 * the first NODEDIRBC value (femModel.cpp:3926-3950), problemType (PROBLEM,
 * femModel.cpp:4036-4050). */
typedef struct fm_poisson_desc {
  int32_t elem_type;             /* FM_TET4 or FM_HEXA8 */
  int32_t problem;               /* FM_POISSON_* */
  int64_t n_nodes, n_elems;
  const double* coords;          /* n_nodes x 3 */
  const int32_t* conn;           /* n_elems x elem_type, 0-based */
  const double* diffusivity;     /* n_elems x 3 */
  int64_t n_sources;
  const int32_t* source_elem;    /* element of each ELSOURCE row */
  const double* source_value;
  int64_t n_neumann;
  const int32_t* neumann_off;    /* n_neumann + 1 offsets into neumann_nodes */
  const int32_t* neumann_nodes;  /* face nodes of each FACENEUMANN row */
  const double* neumann_value;
  int64_t n_dirichlet;
  const int32_t* dir_node;
  const double* dir_value;
} fm_poisson_desc;

typedef struct fm_poisson fm_poisson;

/* Assembles the system on the host (element matrices in parallel, every
 * matrix entry and right-hand-side value summed in element order) and
 * uploads it to `device`.  The descriptor's arrays are copied. */
FM_API int fm_poisson_create(const fm_poisson_desc* desc, int32_t device, fm_poisson** out);
FM_API int fm_poisson_destroy(fm_poisson* s);
/* Preconditioned CG from x = 0 until ||r|| <= rel_tol ||b|| or max_iter
 * iterations; every reduction is summed in a fixed order, so the iterates
 * are the same from run to run.  FM_ERR_DIVERGED if the iteration breaks down
 * (a non-positive curvature or a NaN).  Device time of the solve in
 * *device_ms (may be NULL). */
FM_API int fm_poisson_solve(fm_poisson* s, double rel_tol, int32_t max_iter, int32_t* iterations,
                            double* rel_residual, double* device_ms);
/* The result fields: x (n_nodes; the average subtracted for
 * FM_POISSON_PPE) and, when cell_distance is non-NULL and the problem is
 * FM_POISSON_DISTANCE, the element wall distance (n_elems). */
FM_API int fm_poisson_get_solution(fm_poisson* s, double* x, double* cell_distance);
/* The same from a .dat file: the keywords femPoissonSolver::solve reads
 * (PROBLEM, NODE, ELEMENT, ELDIFF, ELSOURCE, FACENEUMANN, NODEDIRBC;
 * femModel::ReadFromFEMTextFile, femModel.cpp:3719-4213, with its token
 * rules), parsed on the host threads. */
FM_API int fm_poisson_read_dat(const char* path, int32_t device, fm_poisson** out);
/* The results in femModel::ExportToVTKLegacy's legacy-VTK layout
 * (femModel.cpp:1294-1530) as the reference's Poisson driver writes them
 * (src/main.cpp:508-511): mesh with the connectivity the solver used,
 * "PoissonResult", dirBC, neuBC, diffusivity, source and, for
 * FM_POISSON_DISTANCE, "cellDistance".  After fm_poisson_solve. */
FM_API int fm_poisson_write_vtk(fm_poisson* s, const char* path);
/* Sizes of the assembled system: rows and stored matrix entries. */
FM_API int fm_poisson_info(const fm_poisson* s, int64_t* rows, int64_t* nonzeros);
/* The model behind a solver (also one read by fm_poisson_read_dat): node and
 * element counts, element type (FM_TET4 / FM_HEXA8) and FM_POISSON_* problem
 * (femModel's nodeList / elementList sizes and problemType).  Null outputs
 * are skipped. */
FM_API int fm_poisson_model(const fm_poisson* s, int64_t* n_nodes, int64_t* n_elems, int32_t* elem_type,
                            int32_t* problem);

#ifdef __cplusplus
}
#endif
#endif /* FEMORPH_B200_H */
