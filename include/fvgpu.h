/*
 * fvgpu.h — C ABI of the B200 explicit finite-volume step.
 *
 * Plain C types only (no CUDA or torch types): pointers are host pointers
 * unless the name ends in _device, sizes are int64_t, every call returns an
 * fv_status (0 = OK, negative = error; fv_last_error() gives the message).
 * Calls on one fv_solver are not thread-safe; different solvers are
 * independent.  State arrays use fvhyper's layout: AoS q[V*cell + k] over
 * n_total = real cells + boundary ghost cells, reference cell numbering
 * (fvhyper/src/explicit.cpp:665-678).
 *
 * Reference interfaces replaced (paths relative to the fvhyper repository):
 *   fv_mesh_create / fv_mesh_read_msh  <- mesh::read_file          fvhyper/mesh.h:193, src/mesh.cpp:803-855
 *   fv_solver_create (fv_physics)      <- the user's link-time physics symbols
 *                                         (vars, solver:: flags, calc_flux, calc_dt,
 *                                         limiter_func, boundaries::bounds)
 *                                         fvhyper/explicit.h:31-85, fvhyper/mesh.h:36-39
 *   fv_run                             <- run(name, q, pool, m, opt) fvhyper/explicit.h:175-181
 *   fv_run_options                     <- solverOptions              fvhyper/explicit.h:152-160
 *   fv_stage_dt                        <- calc_dt + min_dt           explicit.cpp:729-734, 555-564
 *   fv_stage_gradients_limiters        <- calc_gradients + calc_limiters explicit.cpp:112-258
 *   fv_stage_update                    <- calc_time_derivatives + update_cells + update_bounds
 *                                                                    explicit.cpp:261-417
 *   fv_residuals                       <- calc_residuals             explicit.cpp:481-552
 *   fv_group_create / fv_group_run     <- the MPI run: mesh::read_file of a gmsh partition with
 *                                         make_comms, run() with update_comms, validate_dt and
 *                                         the rank sums of calc_residuals
 *                                         mesh.cpp:574-617, 673-799; explicit.cpp:420-477, 498-550,
 *                                         567-621, 636-648, 729-746
 *   fv_mesh_partition                  <- make_comms' send/receive index lists mesh.cpp:673-799
 */
#ifndef FVGPU_H
#define FVGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    FV_OK = 0,
    FV_ERR_ARG = -1,          /* invalid argument */
    FV_ERR_CUDA = -2,         /* CUDA runtime error (message has the CUDA error string) */
    FV_ERR_MESH = -3,         /* malformed mesh (open face, missing boundary edge, zero area, ...) */
    FV_ERR_UNSUPPORTED = -4,  /* option outside the implemented device physics kinds */
    FV_ERR_NONFINITE = -5,    /* state became non-finite (checked by fv_check_state) */
    FV_ERR_NOMEM = -6,        /* device allocation failed */
    FV_ERR_IO = -7,           /* file could not be read or written */
    FV_ERR_COMM = -8          /* NCCL unavailable or a collective failed (decompositions) */
} fv_status;

/* Physics kinds implemented on the device (see finite-volume-2d-cpp_b200/physics.py). */
/* FV_FLUX_NS: the compressible Navier-Stokes flux of examples/flatPlate and
 * examples/nacaTransient (FV_FLUX_ROE_ST minus the viscous stresses and heat
 * conduction from the face gradient; mu, pr, cp, r below).
 * FV_FLUX_BURGERS_DIFF: FV_FLUX_BURGERS plus -(grad q . n) per variable from
 * the face gradient, the reference's regression-test physics
 * (tests/tests.cpp:76-117, V = 2). */
enum { FV_FLUX_ROE_FS = 1, FV_FLUX_ROE_ST = 2, FV_FLUX_BURGERS = 3, FV_FLUX_DIFFUSION = 4, FV_FLUX_NS = 5,
       FV_FLUX_BURGERS_DIFF = 6 };
enum { FV_LIM_ZERO = 0, FV_LIM_MICHALAK = 1, FV_LIM_VENKAT = 2, FV_LIM_MINMOD = 3 };
/* VISC_MIN (examples/flatPlate/main.cpp:230-277) and VISC_SUM
 * (examples/nacaTransient/main.cpp:234-285): convective + 2 x viscous
 * eigenvalue, min over faces from 1 or summed over faces. */
enum { FV_DT_CONST = 0, FV_DT_CFL_SUM = 1, FV_DT_CFL_MIN_SIGNED = 2, FV_DT_VISC_MIN = 3, FV_DT_VISC_SUM = 4 };
/* NOSLIP: b = (rho, -rho u, -rho v, rho E) (examples/flatPlate/main.cpp:361-366).
 * FARFIELD_B0: FARFIELD with b[2] = b[0]*(...) in the subsonic branches
 * (examples/flatPlate/main.cpp:286-352, nacaTransient/main.cpp:294-360). */
/* TANGENT (V = 2): the fixed state b = (-n_y, n_x) of tests/tests.cpp:132-135. */
enum { FV_BC_COPY = 0, FV_BC_WALL = 1, FV_BC_INLET_OUTLET = 2, FV_BC_FARFIELD = 3, FV_BC_NOSLIP = 4,
       FV_BC_FARFIELD_B0 = 5, FV_BC_TANGENT = 6 };

/* Arithmetic of the step.
 * FP64_EXACT: FP64, the reference's evaluation order, no FMA contraction:
 *             bit-identical to the reference CPU solver.
 * FP64:       FP64 with fused multiply-adds and reciprocal reuse
 *             (<= 1e-12 relative per step against the reference; up to
 *             5e-12 where the residual is a few per cent of the face
 *             fluxes, as in the near-uniform flat-plate flow).
 * FP32:       FP32 bulk flux/gradient/limiter arithmetic; FP64 conserved
 *             state, RK accumulation, residual and force sums. */
enum { FV_PREC_FP64_EXACT = 0, FV_PREC_FP64 = 1, FV_PREC_FP32 = 2 };

typedef struct {
    int32_t V;          /* vars (explicit.h:31): 4 for Euler, 2 for the Burgers kind, 1 for diffusion */
    int32_t flux;       /* FV_FLUX_* */
    int32_t order2;     /* do_calc_gradients && do_calc_limiters && linear_interpolate */
    int32_t limiter;    /* FV_LIM_* (limiter_func) */
    int32_t dt_kind;    /* FV_DT_* (calc_dt) */
    int32_t global_dt;  /* solver::global_dt */
    double gamma;       /* ratio of specific heats */
    double K;           /* limiter constant (explicit.cpp:27 hard-codes 7.5) */
    double cfl;
    double dt_const;
    int32_t n_groups;          /* boundary groups (physical names) */
    const int32_t* group_bc;   /* [n_groups] FV_BC_* per group */
    const double* group_bv;    /* [n_groups*4] far-field/inflow state for INLET_OUTLET/FARFIELD */
    int32_t positivity_guard;  /* not in the reference (0 = the reference's scheme): a MUSCL
                                  face state with rho <= 0 or p <= 0 falls back to the
                                  cell value */
    int32_t diffusive;         /* solver::diffusive_gradients: every stage computes the cell
                                  gradients (no limiter when order2 = 0) and the flux gets
                                  the corrected face gradient of explicit.cpp:70-109.  Used
                                  by FV_FLUX_DIFFUSION (V = 1, order2 = 0, constant dt,
                                  copy boundaries: examples/heatTransfer) and FV_FLUX_NS */
    double mu, pr, cp, r;      /* viscosity, Prandtl number, heat capacity, gas constant of
                                  FV_FLUX_NS and the viscous dt kinds (the examples' consts::) */
    int32_t smooth_residuals;  /* solver::smooth_residuals: two Jacobi sweeps of implicit
                                  residual smoothing (explicit.cpp:32-66) after each stage's
                                  time derivatives, in fv_run; with FV_FLUX_BURGERS_DIFF (the
                                  only physics of the reference that uses it).  The stage-level
                                  entry points do not smooth. */
} fv_physics;

typedef struct {
    uint64_t max_step;        /* solverOptions::max_step */
    double max_time;          /* solverOptions::max_time */
    double tolerance;         /* solverOptions::tolerance */
    uint64_t print_interval;  /* solverOptions::print_interval */
    int32_t n_alpha;          /* RK stages; the reference hard-codes 5 (explicit.cpp:681-687) */
    const double* alpha;      /* [n_alpha] stage coefficients */
    int32_t restart;          /* 1: step = 0, time = 0, fill ghosts first (as run() does);
                                 0: continue from the solver's current step/time/R0 */
    /* Called on the host after each chunk for every print step
       (step % print_interval == 0, and step 0), with the time at the start of
       that step and R normalised as run() prints it.  May be NULL. */
    void (*on_print)(void* user, uint64_t step, double time, const double* R, int32_t V);
    void* user;
} fv_run_options;

typedef struct {
    uint64_t step;     /* steps taken in total */
    double time;       /* accumulated time (time += dt[0], explicit.cpp:800) */
    double R[8];       /* residual norms as run() leaves them */
    double R0[8];      /* step-0 residual norms */
} fv_run_info;

typedef struct fv_mesh fv_mesh;
typedef struct fv_solver fv_solver;

const char* fv_last_error(void);
int fv_version(void);

/* ---- mesh (host) -------------------------------------------------------- */
/* Element mesh -> FV geometry exactly as mesh::read_file builds it
 * (mesh.cpp:821-853): edges in first-visit order, centroids, outward normals,
 * areas, one ghost cell per boundary segment in segment order.
 * cells4: [n_cells][4] node indices, -1 in column 3 for triangles.
 * bnd_nodes: [n_bnd][2]; bnd_group: [n_bnd] group index < n_groups. */
int fv_mesh_create(int64_t n_nodes, const double* nodes_x, const double* nodes_y,
                   int64_t n_cells, const int32_t* cells4, int64_t n_bnd,
                   const int32_t* bnd_nodes, const int32_t* bnd_group, int32_t n_groups,
                   fv_mesh** out);
/* Gmsh MSH 4.1 ASCII file (single partition) -> mesh; boundary groups are
 * the physical names of the boundary curves, in order of first use. */
int fv_mesh_read_msh(const char* path, fv_mesh** out);
/* SU2 native ASCII mesh (2D: triangles, quadrilaterals, segment markers) ->
 * mesh; boundary groups are the marker tags in file order, nodes and cells
 * keep file order.  No counterpart in the reference, whose reader takes Gmsh
 * files only (examples/naca/naca.geo:1-7 converts its SU2 meshes first). */
int fv_mesh_read_su2(const char* path, fv_mesh** out);
/* A batch of independent cases as one mesh (the disjoint union of the case
 * meshes): reference numbering = the real cells of case 0, 1, ..., then the
 * ghosts of case 0, 1, ...; boundary groups are merged by name.  A solver on
 * a batch advances every case in the same launches, each case with its own
 * global dt minimum (min_dt over that case's cells only) and its own time
 * (fv_batch_times).  fv_run's step counter, residual norms (sums over all
 * cases), max_time (checked against case 0's time) and print records are
 * shared by the batch.  No counterpart in the reference, which runs one case
 * per process. */
int fv_mesh_create_batch(int32_t n_cases, const fv_mesh* const* cases, fv_mesh** out);
/* 1 for a single mesh. */
int fv_mesh_case_count(const fv_mesh* m);
/* real_off[n_cases + 1], bound_off[n_cases + 1]: case k's real cells are
 * reference cells [real_off[k], real_off[k+1]), its ghosts are reference
 * cells n_real + [bound_off[k], bound_off[k+1]). */
int fv_mesh_case_offsets(const fv_mesh* m, int64_t* real_off, int64_t* bound_off);
void fv_mesh_destroy(fv_mesh* m);
/* out[5] = {n_nodes, n_real, n_total, n_edges, n_bound} */
int fv_mesh_sizes(const fv_mesh* m, int64_t* out);
int fv_mesh_group_count(const fv_mesh* m);
/* copies group i's name (NUL-terminated, truncated to cap) */
int fv_mesh_group_name(const fv_mesh* m, int32_t i, char* buf, int32_t cap);
/* Reference-numbered geometry (mesh.h:151-171).  Any pointer may be NULL. */
int fv_mesh_geometry(const fv_mesh* m, uint32_t* edge_cells, uint32_t* edge_nodes,
                     double* enx, double* eny, double* elen, double* ecx, double* ecy,
                     double* area, double* ccx, double* ccy, uint32_t* bound_edges,
                     int32_t* bound_group);
/* Element data for output: nodes [n_nodes], cells4 [n_real*4]. */
int fv_mesh_elements(const fv_mesh* m, double* nodes_x, double* nodes_y, int32_t* cells4);
/* Device cell order: new2ref[n_total] (reference index of each device cell). */
int fv_mesh_device_order(const fv_mesh* m, int32_t* new2ref);
/* Host-only inspection of the tile layout a solver builds for tile_cells (64,
 * 128 or 256), in device numbering (no counterpart in the reference; it
 * exposes the data the tile kernels index with).  sizes[5] = n_tiles,
 * max_halo, max_edges, total halo entries, total tile edges.  Each output
 * array may be NULL (call once for the sizes): info [n_tiles][4] = edge
 * offset, edge count, halo offset, halo count; halo [total halo] device cell
 * of each halo slot; edge_ij [total edges] = local i | local j << 16 (owned
 * cell c -> c - tile start, halo slot h -> tile_cells + h); face
 * [4][n_real] = tile-local edge | ghost neighbour << 14 | second cell << 15,
 * 0xFFFF for no face. */
int fv_mesh_tile_layout(const fv_mesh* m, int32_t tile_cells, int64_t* sizes, int32_t* info, int32_t* halo,
                        uint32_t* edge_ij, uint16_t* face);
/* Host-only inspection of the two-ring tile layout of the fused stage
 * kernel (no counterpart in the reference).  sizes[8] = n_tiles, max slots,
 * max gradient slots, max edges (a multiple of 4), max flux edges, total halo
 * entries, total edge entries (each tile's run padded to a multiple of 4),
 * total face-word entries.  Each output array may be NULL: info [n_tiles][8]
 * = edge offset, edge count, flux-edge count, halo offset, ring-1 count,
 * ring-2 count, face offset, 0; halo [total] device cells of ring 1 then
 * ring 2; edge_ij [total] = local i | local j << 16 (owned cell c -> c -
 * tile start, halo slot h -> tile_cells + h); face [total][4] = the face
 * words of each tile's gradient slots (owned, then ring 1), formatted as in
 * fv_mesh_tile_layout. */
int fv_mesh_tile2_layout(const fv_mesh* m, int32_t tile_cells, int64_t* sizes, int32_t* info, int32_t* halo,
                         uint32_t* edge_ij, uint16_t* face);

/* ---- solver (device) ---------------------------------------------------- */
int fv_solver_create(const fv_mesh* m, const fv_physics* ph, int32_t precision, int32_t device,
                     fv_solver** out);
typedef struct {
    int32_t tile_cells;  /* cells per tile = threads per CTA: 64, 128 or 256 (0 = 128) */
    /* Stage kernels of the second-order Euler kinds (Roe fluxes, no
     * diffusive terms, no residual smoothing):
     * FV_STAGE_AUTO (0): where the physics allow the fused kernel,
     *   FV_STAGE_HYBRID in FP32 and FV_STAGE_FUSED in FP64 and FP64_EXACT (and
     *   with the work-list schedule); otherwise FV_STAGE_SPLIT.
     * FV_STAGE_SPLIT (1): a gradient + limiter kernel and a flux + update
     *   kernel per stage (the first stage's gradient kernel also computes dt).
     * FV_STAGE_FUSED (2): one fused kernel per RK stage (gradients, limiter,
     *   fluxes, update, ghost fill) over two-ring tiles, plus one time-step
     *   kernel per step; FV_ERR_UNSUPPORTED when the physics do not allow it.
     * FV_STAGE_HYBRID (3): the split kernels for the first stage of each step
     *   (whose gradient kernel also computes dt, so the step has no separate
     *   time-step kernel) and the fused kernel for the others; not with the
     *   work-list schedule.  All four give the same results (bit for bit in
     *   FP64_EXACT). */
    int32_t stage_kernels;
    /* Schedule of the fused stage kernel: FV_SCHED_TILE (0) one CTA of one
     * thread per cell per tile; FV_SCHED_WORKLIST (1) as many CTAs as the
     * device holds at once, each taking the next tile from a per-stage work
     * list; FV_SCHED_TILE2 (2) one CTA of two threads per cell per tile
     * (tiles of at most 128 cells), so the gradient and flux phases of a
     * tile run in one pass.  Ignored for the split kernels. */
    int32_t schedule;
} fv_solver_options;
enum { FV_STAGE_AUTO = 0, FV_STAGE_SPLIT = 1, FV_STAGE_FUSED = 2, FV_STAGE_HYBRID = 3 };
enum { FV_SCHED_TILE = 0, FV_SCHED_WORKLIST = 1, FV_SCHED_TILE2 = 2 };
int fv_solver_create_ex(const fv_mesh* m, const fv_physics* ph, int32_t precision, int32_t device,
                        const fv_solver_options* opt, fv_solver** out);
/* Autotuned creation: builds the solver with each tile size (64, 128, 256
 * cells per tile = threads per CTA) and, where the physics allow the fused
 * stage kernel, with each edge-tile layout (split gradient and flux kernels
 * over one-ring tiles, or the fused kernel over two-ring tiles); times
 * n_steps steps of the given RK stages from state q on the device for each
 * candidate (after one untimed step that captures the step graph), the
 * fused kernel with both schedules, and keeps the fastest.  The returned
 * solver holds state q again, step 0; tile_cells and ms_per_step (may be
 * NULL) report the choice, fv_solver_stage_kernels and fv_solver_schedule
 * the layout and schedule. */
int fv_solver_create_tuned(const fv_mesh* m, const fv_physics* ph, int32_t precision, int32_t device,
                           const double* q, const double* alpha, int32_t n_alpha, int32_t n_steps,
                           fv_solver** out, int32_t* tile_cells, double* ms_per_step);
int fv_solver_destroy(fv_solver* s);

/* ---- domain decomposition (one process per GPU, NCCL between processes) ----
 * The mesh's real cells are split into n_parts contiguous ranges of the
 * solver's cell order (a Hilbert order, so parts are compact).  Each part
 * holds its cells, two rings of halo cells and the boundary ghosts of the
 * first ring, and after every RK stage receives the stage states of its halo
 * cells from their owners (the reference exchanges q, gx, gy, limiters and dt
 * of one ring per stage; with two rings each part recomputes the ring-1
 * gradients and limiters itself, so only the stage state moves).  The time
 * step is the minimum over all parts (min_dt over the whole mesh; the
 * reference's validate_dt, explicit.cpp:567-621, keeps the minimum of rank 0
 * and the last rank only) and the residual norms sum every part's partial
 * sums in one order on every process, so all parts and processes take the
 * same steps.  The state of every cell equals the single-solver state bit
 * for bit; R differs in summation order only.
 * Physics: first order, or second order with the fused stage kernel (the
 * Roe kinds); not the diffusive kinds or residual smoothing
 * (FV_ERR_UNSUPPORTED), not batches of cases. */
typedef struct fv_group fv_group;
enum { FV_EXCHANGE_COPY = 0, FV_EXCHANGE_P2P = 1 };
typedef struct {
    int32_t n_parts;        /* parts of the decomposition, >= 1, a multiple of n_ranks */
    int32_t rank, n_ranks;  /* this process and the number of processes; process r holds
                               parts [r * n_parts / n_ranks, (r + 1) * n_parts / n_ranks) */
    const void* nccl_id;    /* 128-byte id from fv_group_nccl_id on one process, passed to
                               all (NULL when n_ranks == 1) */
    int32_t nccl_local;     /* 1: parts of this process also exchange through NCCL (to
                               itself) instead of device copies */
    fv_solver_options solver;  /* every part's tile size, stage kernels and schedule */
    int32_t serial_exchange;   /* 0 (default): with the fused stage kernel and one CTA per
                                  tile, each part's cells that other parts read come first;
                                  their tiles and then the halo exchange run on a second,
                                  high-priority stream while the remaining tiles compute.
                                  1: the exchange follows all tiles of the stage. */
    int32_t transport;         /* halo states between parts: FV_EXCHANGE_COPY (0) NCCL
                                  send/recv between processes (packed, then unpacked) and
                                  device reads within one; FV_EXCHANGE_P2P (1) stored straight
                                  into the reading part's stage buffer (peer memory through
                                  CUDA IPC between processes) by the fused stage launch that
                                  computes them (a push kernel after first-order stages), which
                                  then releases an epoch flag there; the reader waits for it (a
                                  bounded poll) before reading them */
    int64_t wait_polls;        /* P2P: polls of one halo wait before it gives up (0 = 2^24) */
    double timeout_ms;         /* with NCCL: the longest wait for one chunk of steps (0 = 300 s).
                                  A chunk that makes no progress within it, or an NCCL error,
                                  aborts the communicator and fv_group_run returns FV_ERR_COMM
                                  (the group cannot run again). */
} fv_group_options;
int fv_group_nccl_id(void* id128);
/* Collective over the n_ranks processes (each passes the whole mesh, its rank
 * and the same n_parts and id). */
int fv_group_create(const fv_mesh* m, const fv_physics* ph, int32_t precision, int32_t device,
                    const fv_group_options* o, fv_group** out);
int fv_group_destroy(fv_group* g);
/* q: the whole mesh's state in reference numbering, AoS [n_total][V].  get
 * writes the cells and boundary ghosts this process's parts own and leaves
 * the rest of q as it was. */
int fv_group_set_state(fv_group* g, const double* q);
int fv_group_get_state(fv_group* g, double* q);
/* fv_run for the decomposition (collective): same options and results. */
int fv_group_run(fv_group* g, const fv_run_options* opt, fv_run_info* info);
/* out[8]: local parts, owned real cells, halo cells received per stage,
 * cells sent per stage, tiles, 1 if an NCCL communicator exists, band tiles
 * (computed before the exchange; -1 when the exchange follows all tiles),
 * the transport in use (FV_EXCHANGE_*) */
int fv_group_info(fv_group* g, int64_t* out);
int fv_group_last_run_stats(fv_group* g, double* device_ms, int64_t* kernel_launches);
/* Host-only: the plan of part `part` of n_parts.  sizes[11]: local real cells,
 * local cells (with ghosts), local edges, owned real cells, owned ghosts,
 * local index of reference cell 0 (-1 if another part owns it), the part
 * that owns it, cells received and cells sent per stage, local ghosts, owned
 * cells in other parts' halos (the band: local cells [0, band)).
 * fv_mesh_partition fills (each may be NULL): local2ref [local cells]
 * reference index of each local cell (owned cells, halo cells, owned ghosts,
 * halo ghosts); local_edges [local edges] reference index of each local edge;
 * recv_off [n_parts + 1] / recv_idx: local cells whose states come from part
 * r; send_off [n_parts + 1] / send_idx: local cells sent to part r, in r's
 * receive order. */
int fv_mesh_partition_sizes(const fv_mesh* m, int32_t n_parts, int32_t part, int64_t* sizes);
int fv_mesh_partition(const fv_mesh* m, int32_t n_parts, int32_t part, int32_t* local2ref, int32_t* local_edges,
                      int64_t* recv_off, int32_t* recv_idx, int64_t* send_off, int32_t* send_idx);

/* cudaStream_t as void*; NULL = the solver's own stream */
int fv_solver_set_stream(fv_solver* s, void* stream);
int fv_solver_sync(fv_solver* s);
/* State in reference numbering, AoS [n_total][V]. */
int fv_set_state(fv_solver* s, const double* q);
int fv_get_state(fv_solver* s, double* q);
int fv_set_state_device(fv_solver* s, const double* q_device);
int fv_get_state_device(fv_solver* s, double* q_device);
/* The run() time loop on the device (explicit.cpp:708-801).  Steps are
 * captured in CUDA graphs of `chunk` steps; stopping criteria are evaluated
 * on the device, so the host only waits once per chunk. */
int fv_run(fv_solver* s, const fv_run_options* opt, fv_run_info* info);
/* Continue a run in another solver of the same mesh, typically with another
 * precision (FP32-bulk for the transient, FP64 for the tail of a steady
 * solve, whose residual drop FP32 flux arithmetic cannot take below about
 * 1e-5): copies src's state and run control (step, time, R0, R) into dst, so
 * fv_run(dst, restart = 0) carries on with the same step count, time and
 * residual normalisation.  Both solvers must be on one device.  No
 * counterpart in the reference (explicit.cpp:657-817 runs in one precision). */
int fv_solver_continue_from(fv_solver* dst, fv_solver* src);
/* Per-ghost boundary states: bv[n_bound][4] (reference ghost order) replaces
 * the group state of INLET_OUTLET / FARFIELD ghosts, e.g. an inflow profile
 * that varies along the inlet.  NULL restores the group states.  The
 * reference binds one boundary function per physical name (mesh.cpp:662-667);
 * a varying inflow there needs one function per inlet segment. */
int fv_solver_set_ghost_states(fv_solver* s, const double* bv);
/* times[n_cases]: each case's accumulated time (time += that case's dt[0]). */
int fv_batch_times(fv_solver* s, double* times);
/* R after the last step (sqrt of sum qt^2 A over real cells, un-normalised). */
int fv_residuals(fv_solver* s, double* R);
/* Returns FV_ERR_NONFINITE if any real-cell state is NaN/Inf, or if an
 * Euler state has rho <= 0 or p <= 0. */
int fv_check_state(fv_solver* s);
/* Pressure force on the faces of boundary group `group` (FP64 sum over the
 * group's faces of p(interior state) * n * length). */
int fv_boundary_force(fv_solver* s, int32_t group, double* fx, double* fy);
/* Chunk length of the captured step graphs (default 16). */
int fv_solver_set_chunk(fv_solver* s, int32_t steps);
/* out[6] = {tiles, cells per tile, max halo cells per tile, max edges per
 * tile, precision, bytes per stored stage value}. */
int fv_solver_info(fv_solver* s, int64_t* out);
/* Extra output fields evaluated on the device (the writeVtk callbacks of
 * post.cpp:165-188): for each of n_fields (at most 8) kinds FV_OUT_*, the
 * values of the real cells in reference order, one after the other in `out`
 * (n_real values for a one-component kind, n_real pairs for a two-component
 * one).  q: a host state [n][V] in reference numbering, n = n_real or
 * n_total; NULL evaluates the solver's current state.  gamma is the
 * solver's.  Bit-identical to fv_kind_output cell by cell. */
int fv_output_fields(fv_solver* s, const double* q, int64_t n, int32_t n_fields, const int32_t* kinds,
                     double* out);
/* The stage kernels the solver runs: FV_STAGE_FUSED or FV_STAGE_SPLIT. */
int fv_solver_stage_kernels(fv_solver* s);
/* The fused kernel's schedule: FV_SCHED_TILE, FV_SCHED_WORKLIST or FV_SCHED_TILE2. */
int fv_solver_schedule(fv_solver* s);
/* Device time of the last fv_run's chunks and per-kernel launch count. */
int fv_last_run_stats(fv_solver* s, double* device_ms, int64_t* kernel_launches);

/* Per-kernel device timing: runs n_steps more time steps without graph
 * capture, with a CUDA event after every kernel on the solver's stream.
 * out_ms[6] / out_count[6] per kernel kind: 0 step control, 1 time step,
 * 2 gradients + limiters, 3 flux + update + ghost fill, 4 step end, 5 the
 * fused stage kernel (gradients through ghost fill in one launch). */
int fv_profile_kernels(fv_solver* s, const double* alpha, int32_t n_alpha, int32_t n_steps,
                       double* out_ms, int64_t* out_count);

/* ---- stage-level entry points (host arrays, reference numbering) -------- */
/* dt per cell [n_total]; global_min applies min_dt (explicit.cpp:555-564). */
int fv_stage_dt(fv_solver* s, const double* q, double* dt, int32_t global_min);
/* gx, gy, lim [n_total*V] from the fused gradient + limiter kernel.
 * FP64_EXACT: the reference's gx, gy and limiters.  FP64 / FP32: these modes
 * keep the limiter multiplied into the gradients, so gx, gy receive gx*lim,
 * gy*lim and lim is filled with 1. */
int fv_stage_gradients_limiters(fv_solver* s, const double* q, double* gx, double* gy,
                                double* lim);
/* One RK stage from the fused flux + update + ghost-fill kernel (FP64 / FP32:
 * gx, gy are the limited gradients and lim is ignored):
 * q_out = q_base + qt(q_stage) * dt * alpha on real cells, then the ghost
 * fill from q_out with the given gx, gy, lim (explicit.cpp:742-745).
 * dt [n_total].  q_out [n_total*V]. */
int fv_stage_update(fv_solver* s, const double* q_base, const double* q_stage,
                    const double* gx, const double* gy, const double* lim, const double* dt,
                    double alpha, double* q_out);
/* fv_stage_dt without any device allocation.  No counterpart in the
 * reference: it exists for callers that cannot call cudaMalloc -- code that
 * embeds this solver in a loop whose GPU memory is fully reserved up front
 * by the host application's own pool, or that must not pay the implicit
 * device synchronisation of an allocation between its queued kernels.
 * q_device: [n_total][V] state, dt_device: [n_total] output, both device
 * memory in reference numbering.  Work is queued on `stream` (NULL = the
 * solver's stream) and is complete when that stream is; nothing is copied
 * to the host.  Its working arrays are one fixed 8 MiB device array per GPU
 * (held until the process exits), so meshes needing more (about 200k cells
 * in FP64, 150k in FP32) are rejected with FV_ERR_ARG.  The first call on a
 * device looks up that array's device address; make it before any stream
 * capture.  The address is kept for the rest of the process: after a
 * cudaDeviceReset (or anything else that tears down the device's primary
 * context) it is stale, so do not call this entry point again in that
 * process.  All calls share the array: calls that overlap on the GPU (two
 * streams, two threads) race and must be serialised by the caller. */
int fv_stage_dt_noalloc(fv_solver* s, const double* q_device, double* dt_device, int32_t global_min,
                        void* stream);
/* Ghost fill alone (explicit.cpp:380-417) on q (in place). */
int fv_stage_bounds(fv_solver* s, double* q, const double* gx, const double* gy,
                    const double* lim);

/* ---- host evaluation of the device physics kinds ------------------------ */
/* The device kinds' arithmetic run on the host (bit-identical to the device's
 * FP64_EXACT mode and to the reference example functions each kind restates).
 * The fvhyper shim compares a user's calc_flux / limiter_func /
 * boundaries::bounds entries with these on probe states to choose the kind
 * (explicit.h:53,71-78; mesh.h:36-39).  n = {nx, ny}. */
int fv_kind_flux(int32_t flux, double gamma, const double* qi, const double* qj, const double* n,
                 double* f);
/* calc_flux with its face gradient arguments (explicit.h:71-78): gx, gy are
 * the [V] face gradients the reference passes; the non-diffusive kinds
 * ignore them.  Reads ph->flux, V, gamma and (FV_FLUX_NS) mu, pr, cp, r. */
int fv_kind_flux_grad(const fv_physics* ph, const double* qi, const double* qj, const double* gx,
                      const double* gy, const double* n, double* f);
/* gradient_for_diffusion (explicit.cpp:70-109): the corrected face gradient
 * [V] from the cell gradients, cell states and centroids ci, cj ([2] each). */
int fv_kind_face_gradient(int32_t V, const double* gxi, const double* gyi, const double* gxj,
                          const double* gyj, const double* qi, const double* qj, const double* ci,
                          const double* cj, double* gxf, double* gyf);
int fv_kind_limiter(int32_t kind, double y, double* out);
/* Extra output fields of the examples' post::extra_scalars / extra_vectors
 * callbacks (post.h:24-30): FV_OUT_PRESSURE and FV_OUT_MACH (one component,
 * examples/forwardStep/main.cpp:289-299), FV_OUT_VELOCITY (u, v;
 * forwardStep/main.cpp:283-287) and FV_OUT_STATE01 (q[0], q[1];
 * examples/burgers/main.cpp:133-137), in the examples' arithmetic.  Host copy
 * for identification: returns the number of components written to out. */
enum { FV_OUT_PRESSURE = 1, FV_OUT_MACH = 2, FV_OUT_VELOCITY = 3, FV_OUT_STATE01 = 4 };
int fv_kind_output(int32_t kind, double gamma, const double* q, double* out);
/* bv: [4] boundary state of INLET_OUTLET / FARFIELD (may be NULL otherwise). */
int fv_kind_bc(int32_t kind, int32_t V, double gamma, const double* bv, const double* q,
               const double* n, double* b);

/* ---- discrete adjoint (FP64) ------------------------------------------- */
/* Reverse mode of fv_run's FP64_EXACT time loop for an inflow-parameter
 * problem (no counterpart in the reference):
 *   theta = (M, delta_1 .. delta_nb): the initial state is the free stream
 *   (rho_inf, u = M, v = 0, p_inf), rho_inf and p_inf from param_group's
 *   boundary state; every INLET_OUTLET / FARFIELD ghost gets the state
 *   (rho, rho M, 0, p_inf/(gamma-1) + rho M^2/2) with rho = rho_inf (1 + delta_b)
 *   on param_group faces whose centre y falls in bin b of [bin_lo, bin_hi),
 *   rho = rho_inf elsewhere;
 *   loss = sum over the n_steps steps of dt_n * sum over loss_group faces of
 *   p(interior cell at the step's start) * face length.
 * The forward run keeps the state every checkpoint_every steps; the reverse
 * sweep recomputes each segment, keeping every stage's state, gradients and
 * limiters, and runs the adjoint kernels stage by stage backwards (Roe flux,
 * MUSCL reconstruction, gradients and limiter, ghost fills, RK update, the
 * global CFL time step and the loss).  Needs V = 4, a Roe flux kind and a
 * global CFL-sum or constant time step. */
typedef struct fv_adjoint fv_adjoint;
typedef struct {
    int32_t n_steps;
    int32_t checkpoint_every;
    int32_t n_alpha;          /* RK stages (<= 8) */
    const double* alpha;
    int32_t loss_group;
    int32_t param_group;
    int32_t n_bins;
    double bin_lo, bin_hi;
} fv_adjoint_options;
int fv_adjoint_create(const fv_mesh* m, const fv_physics* ph, int32_t device, const fv_adjoint_options* o,
                      fv_adjoint** out);
/* loss (may be NULL); grad[1 + n_bins] = dL/dtheta, or NULL for the forward
 * run alone (the loss). */
int fv_adjoint_run(fv_adjoint* a, const double* theta, double* loss, double* grad);
/* State after the last forward run, reference numbering [n_total][4]. */
int fv_adjoint_final_state(fv_adjoint* a, double* q);
int fv_adjoint_destroy(fv_adjoint* a);

#ifdef __cplusplus
}
#endif
#endif
