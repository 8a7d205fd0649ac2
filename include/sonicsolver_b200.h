/*
 * sonicsolver_b200.h -- C ABI of the B200 (sm_100a) explicit Euler provider.
 *
 * One opaque solver handle per structured grid (or one batch / server handle
 * for many grids) carries device-resident conserved state and runs the
 * density-based explicit path of sonicSolver on one GPU:
 *   characteristic WENO/TENO reconstruction -> Steger-Warming / Rusanov /
 *   Lax-Friedrichs / Roe / Lax-Wendroff face flux ->
 *   conservative divergence -> ghost/periodic fill -> forwardEuler / SSPRK3 /
 *   classicalRK4 stage combination, with the CFL time step reduced on device.
 *
 * Every entry point returns an int status (SFG_OK = 0) and never exits or
 * throws across the ABI; sfg_last_error() gives the message of the last
 * failure on the calling thread.  Plain pointers and sizes only.
 *
 * Reference interfaces replaced (paths inside the sonicSolver source tree):
 *   - divDispatch(Field&, FluxField&, Residual&, ConvectionScheme, FluxSplitter,
 *     double, IBMBoundaryScheme, int, double, const Model&)
 *       src/solver/discretization/convection/SF_div.h:212-243
 *   - Time::Explicit::begin / executeStage / forwardEuler
 *       src/solver/algorithm/time/SF_explicit.h:47-69,
 *       src/solver/algorithm/time/SF_explicit.cpp:282-530
 *   - RusanovEOS::deltaT(const Field&, const Model&, double)
 *       src/methods/numerics/Flux/SF_rusanovEOS.h:36-38
 *   - Runtime::globalMinimum (MPI_Allreduce MIN of dt)
 *       src/infrastructure/execution/SF_executionRuntime.cpp:126
 *   - Boundary::Applicator::apply(Field&) for zeroGradient ends and the
 *     (declared, unimplemented) periodic interface
 *       src/solver/boundary/SF_applicator.h:51-83
 *   - the flow.conservative op bindings FlowStepPrepare / FlowDtCompute /
 *     FlowStepBegin / ExplicitStageExecute / FlowStepCommit
 *       src/solver/algorithm/SF_flowOperations.cpp:466-522
 */
#ifndef SONICSOLVER_B200_H
#define SONICSOLVER_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes --------------------------------------------------- */
enum {
    SFG_OK = 0,
    SFG_ERR_ARG = 1,          /* invalid argument / unsupported combination   */
    SFG_ERR_CUDA = 2,         /* CUDA runtime failure (message has the text)  */
    SFG_ERR_STATE = 3,        /* rho <= 0, p <= 0 or non-finite state / flux  */
    SFG_ERR_TENO_CUTOFF = 4,  /* TENO5 rejected all three sub-stencils        */
    SFG_ERR_NOMEM = 5,        /* device allocation failed                     */
    SFG_ERR_BUDGET = 6,       /* HBM budget of a batch / server exceeded      */
    SFG_ERR_TIMEOUT = 7,      /* a bounded wait gave up                       */
    SFG_ERR_NOT_FOUND = 8,    /* unknown slot / request id                    */
    SFG_ERR_CANCELLED = 9     /* request was cancelled                        */
};

/* Device status-word bits (sfg_status_word). */
enum {
    SFG_FLAG_NONFINITE = 1u << 0,
    SFG_FLAG_DENSITY = 1u << 1,
    SFG_FLAG_PRESSURE = 1u << 2,
    SFG_FLAG_TENO_CUTOFF = 1u << 3,
    SFG_FLAG_ROE_SOUND = 1u << 4
};

/* ---- recipe identifiers --------------------------------------------- */
/* Convection recipes: the values of FDM::TermRecipeId
 * (src/core/config/types/SF_termRecipe.h:52-64). */
enum {
    SFG_RECIPE_WENO3_STEGER = 0,      /* Steger-Warming, Lax-Friedrichs and     */
    SFG_RECIPE_WENO3_RUSANOV = 1,     /* Lax-Wendroff faces: FP64 single-grid   */
    SFG_RECIPE_WENO3_LAXF = 2,        /* solvers only (SFG_PREC_FP32_FLUX and   */
    SFG_RECIPE_WENO3_ROE = 3,         /* batches take Rusanov and Roe)          */
    SFG_RECIPE_WENO3_LAXW = 4,
    SFG_RECIPE_WENO5_STEGER = 5,
    SFG_RECIPE_WENO5_RUSANOV = 6,
    SFG_RECIPE_WENO5_LAXF = 7,
    SFG_RECIPE_WENO5_ROE = 8,
    SFG_RECIPE_WENO5_LAXW = 9,
    SFG_RECIPE_TENO5_STEGER = 10,
    SFG_RECIPE_TENO5_RUSANOV = 11,
    SFG_RECIPE_TENO5_LAXF = 12,
    SFG_RECIPE_TENO5_ROE = 13,
    SFG_RECIPE_TENO5_LAXW = 14,
    SFG_RECIPE_WENO7_STEGER = 15,
    SFG_RECIPE_WENO7_RUSANOV = 16,
    SFG_RECIPE_WENO7_LAXF = 17,
    SFG_RECIPE_WENO7_ROE = 18,
    SFG_RECIPE_WENO7_LAXW = 19
};
/* Time recipes: the values of FDM::TimeRecipeId (SF_timeRecipe.h:11). */
enum { SFG_TIME_FORWARD_EULER = 0, SFG_TIME_SSPRK3 = 1, SFG_TIME_CLASSICAL_RK4 = 2 };
/* Arithmetic of the reconstruction and face flux.  The conserved state, the
 * stage accumulation, the conserved totals and the dt reduction are FP64 in
 * both modes. */
enum { SFG_PREC_FP64 = 0, SFG_PREC_FP32_FLUX = 1 };
/* Boundary laws per axis end. */
enum {
    SFG_BC_TRANSMISSIVE = 0,  /* zeroGradient: boundary node copies its inner
                                 neighbour and is not advanced; ghosts copy it
                                 (reconstruction/linear/SF_zeroGradient.cpp:88-105) */
    SFG_BC_PERIODIC = 1,      /* ghosts wrap; every node is advanced (the
                                 reference declares PatchBoundaryKind::Periodic,
                                 SF_meshInterface.h:14, but never implements it) */
    SFG_BC_FROZEN = 2,        /* a patch with no boundary condition: the
                                 boundary node is advanced and the ghosts keep
                                 the values they were initialised with, the
                                 boundary node's value at upload (or the
                                 Field layout's first ghost layer)
                                 (SF_applicator.h:162-187 with no BC for the
                                 set; SF_mesh.cpp:544).  Single-grid solvers
                                 only. */
    SFG_BC_LAW = 3            /* physical boundary laws per field (density,
                                 velocity, pressure with the energy rebuilt
                                 from pressure), set by sfg_set_boundary_law;
                                 default: zeroGradient for all three.  The
                                 boundary node is written by the laws and not
                                 advanced; every ghost layer is derived from
                                 it (Boundary::Applicator::apply,
                                 SF_applicator.h:51-83).  Single-grid solvers
                                 only; needs >= 3 nodes on the axis. */
};
/* Law of one field at a SFG_BC_LAW end (BCType of SF_valueTypes.h:28). */
enum {
    SFG_LAW_ZERO_GRADIENT = 0,  /* SF_zeroGradient.cpp:88-131               */
    SFG_LAW_FIXED_VALUE = 1,    /* SF_fixedValue.cpp:110-160                */
    SFG_LAW_SYMMETRY = 2        /* SF_symmetry.cpp:78-136 (velocity: normal
                                   component 0 on the boundary, mirrored in
                                   the ghosts; density, pressure:
                                   zeroGradient)                            */
};
/* Host array layouts for upload / download. */
enum {
    SFG_LAYOUT_NODES = 0,     /* AoS [k][j][i][v] over the nodes only          */
    SFG_LAYOUT_FIELD = 1      /* reference Field storage: AoS [k][j][i][v] with
                                 ng ghost layers on every axis
                                 (src/core/field/SF_field.h:58-67)            */
};

/* ---- descriptors ---------------------------------------------------- */
typedef struct {
    int dim;          /* active axes: the first `dim` of (x, y, z), 1..3      */
    int n[3];         /* nodes per axis (1 on inactive axes)                 */
    double h[3];      /* node spacing; inactive axes: slab thickness          */
    int bc_lo[3];     /* SFG_BC_* per axis, low end                           */
    int bc_hi[3];     /* SFG_BC_* per axis, high end                          */
} sfg_grid_desc;

/* The three laws of one SFG_BC_LAW end (the density / velocity / pressure
 * BCSetting of one patch, FDM::BoundaryConfig); values are read by the
 * fixedValue laws. */
typedef struct {
    int rho;                  /* SFG_LAW_* of density                        */
    int velocity;             /* SFG_LAW_* of velocity                       */
    int pressure;             /* SFG_LAW_* of pressure                       */
    int reserved;             /* 0                                           */
    double rho_value;         /* kg/m3                                       */
    double velocity_value[3]; /* m/s                                         */
    double pressure_value;    /* Pa                                          */
} sfg_boundary_law;

typedef struct {
    int recipe;       /* SFG_RECIPE_*                                        */
    int time_recipe;  /* SFG_TIME_*                                          */
    int precision;    /* SFG_PREC_*                                          */
    double gamma;     /* perfect-gas ratio of specific heats                 */
    double cfl;       /* CFL number of RusanovEOS::deltaT                     */
    double max_dt;    /* numerics maxDeltaT (<= 0: unlimited)                 */
} sfg_numerics_desc;

typedef struct {
    int64_t steps;            /* steps taken                                 */
    double time;              /* physical time reached                       */
    double last_dt;           /* last step size                              */
    double device_ms;         /* device time of the advance (CUDA events)     */
    uint32_t status_bits;     /* SFG_FLAG_* seen                             */
    uint64_t teno_cut;        /* TENO5 sub-stencils cut (when counted)        */
    uint64_t teno_cores;      /* TENO5 cores evaluated (when counted)         */
} sfg_stats;

typedef struct sfg_solver_s* sfg_solver;

/* ---- errors and version --------------------------------------------- */
const char* sfg_last_error(void);
int sfg_version(int* major, int* minor);
/* Recipe name as the case.yaml token (e.g. "weno5Rusanov"); NULL if unknown.
 * Names of FDM::toString(TermRecipeId), SF_termRecipe.h:242-259. */
const char* sfg_recipe_name(int recipe);
/* Recipe id from its case.yaml token; SFG_ERR_ARG if not provided here. */
int sfg_recipe_from_name(const char* name, int* recipe);

/* ---- single grid ------------------------------------------------------ */
/* Binds the provider to the current CUDA device and allocates the state.
 * `stream` is a cudaStream_t (NULL: the solver creates its own). */
int sfg_create(const sfg_grid_desc* grid, const sfg_numerics_desc* numerics,
               void* stream, sfg_solver* out);
int sfg_destroy(sfg_solver s);
/* Ghost layers of the reference Field layout (3 for WENO5/TENO5). */
int sfg_ghost_layers(sfg_solver s, int* ng);
/* Number of doubles of a host array in `layout`. */
int sfg_state_size(sfg_solver s, int layout, size_t* count);
/* Laws of a SFG_BC_LAW end (axis 0..dim-1, end 0 = low, 1 = high).  They
 * act from the next step on, where the reference applies its boundary
 * conditions: at the start of every step (FlowStepPrepare, in sfg_step and
 * sfg_advance), before every stage's RHS and after a step's last stage
 * (FlowStepCommit).  A host plan that drives sfg_stage itself calls
 * sfg_apply_boundary for FlowStepPrepare.  Boundary nodes on two or more
 * law faces (box edges and corners) are read by no stencil of a solved node
 * and are not maintained. */
int sfg_set_boundary_law(sfg_solver s, int axis, int end, const sfg_boundary_law* law);
/* Applies the laws of every SFG_BC_LAW end to the current state once (the
 * reference's Boundary::Applicator::apply on the Field). */
int sfg_apply_boundary(sfg_solver s);
/* Curvilinear grids: the per-node metrics of the reference Field, 10 doubles
 * per node in the order Jac (= 1/J), XiX, XiY, XiZ, EtX, EtY, EtZ, ZeX, ZeY,
 * ZeZ (src/core/field/SF_field.h metric arrays; computed by the mesh,
 * src/infrastructure/mesh/SF_mesh.cpp:260-339), in SFG_LAYOUT_NODES (AoS over
 * the nodes) or SFG_LAYOUT_FIELD (AoS with the ghost layers; a frozen end's
 * ghost face reads them).  From then on every face takes the cofactor
 * 0.5 (m_i / Jac_i + m_i+1 / Jac_i+1) as normal and area
 * (SF_canonicalFace.h:56-118), the residual is Jac_node * sum_d dF_d, and the
 * CFL rate uses the node's metric vectors; the grid's h[] is no longer read
 * by the operator.  FP64 with all fluxes but Lax-Wendroff (which needs node
 * coordinates); FP32-flux with Rusanov and Roe. */
int sfg_set_metrics(sfg_solver s, const double* metrics, int layout);
/* Host <-> device copies of the conserved state (pageable or pinned host
 * memory; synchronous with respect to the solver's stream). Upload resets the
 * time to `time`. */
int sfg_upload(sfg_solver s, const double* host, int layout, double time);
int sfg_download(sfg_solver s, double* host, int layout);
/* Resume: sfg_upload plus the step counter (the time and step count that
 * sfg_time reported when the state was downloaded).  A run downloaded
 * between two steps and restored into a solver with the same grid, numerics
 * and metrics continues with the same dt sequence and the same bits as the
 * run that was never interrupted: between steps the device keeps nothing
 * but the state and the clock, and the CFL minimum is recomputed from the
 * state.  The reference restarts from a state file and the case's start
 * time (CheckpointIO::read, src/infrastructure/io/checkpoint/SF_checkpoint.h:6;
 * initializeSingleFluidRestart, src/models/physics/fluidStateModel/
 * SF_factory.h:137-150). */
int sfg_restore(sfg_solver s, const double* host, int layout, double time, int64_t steps);
/* The same from / to device memory (AoS node layout, no ghosts). */
int sfg_upload_device(sfg_solver s, const double* dev_nodes_aos, double time);
int sfg_download_device(sfg_solver s, double* dev_nodes_aos);

/* FlowDtCompute: CFL step of the current state, min'ed with max_dt and
 * `limit` (<= 0: no limit).  Reduced on device; copied to *dt. */
int sfg_compute_dt(sfg_solver s, double limit, double* dt);
/* FlowStepBegin + ExplicitStageExecute(stage) + (after the last stage)
 * FlowStepCommit, at the given dt.  stage 0 snapshots q0. */
int sfg_stage(sfg_solver s, int stage, double dt);
/* All stages of one step of size dt (dt <= 0: the CFL step, clipped to
 * `limit` when limit > 0). Advances the solver time. */
int sfg_step(sfg_solver s, double dt, double limit);
/* Time::Driver loop: steps until t_end (or max_steps), clipping dt at
 * t_end and at every multiple of write_interval (<= 0: none).  Runs without
 * host synchronisation inside a CUDA graph of `graph_steps` steps
 * (<= 0: default).  dt_out (may be NULL) receives up to dt_capacity dts. */
int sfg_advance(sfg_solver s, double t_end, int64_t max_steps, double write_interval,
                int graph_steps, double* dt_out, int64_t dt_capacity, sfg_stats* stats);
/* Spatial residual R = Jac * sum_d dF_d of the current state (node layout,
 * AoS; unsolved boundary nodes are 0) -- operator-level parity. */
int sfg_residual(sfg_solver s, double* host_nodes_aos);
/* Stage combination alone with a caller-supplied residual (node layout AoS):
 * stage arithmetic parity.  Updates the state as sfg_stage would. */
int sfg_stage_with_residual(sfg_solver s, int stage, double dt, const double* host_residual);
/* Conserved totals sum_nodes Q_v * cell volume (FP64), v = 0..4. */
int sfg_conserved_totals(sfg_solver s, double totals[5]);
int sfg_time(sfg_solver s, double* time, int64_t* steps);
/* Device status word (SFG_FLAG_* bits) accumulated since the last clear. */
int sfg_status_word(sfg_solver s, uint32_t* bits, int clear);
/* TENO5 cut-off accounting (enable = 1 adds counters to the kernels). */
int sfg_set_counting(sfg_solver s, int enable);
int sfg_get_counters(sfg_solver s, uint64_t* teno_cores, uint64_t* teno_cut);

/* ---- batches of independent grids ---------------------------------------
 * Many 1-D / 2-D grids of uneven sizes, each with its own CFL step, end time
 * and status, advanced together: per batch step one persistent kernel
 * computes every grid's CFL minimum, one persistent kernel per stage works
 * through a list of tiles of all grids, and a per-grid clock update follows;
 * runs of steps execute as one CUDA graph.  Grids can be added and removed
 * between calls without rebuilding the graph (continuous batching).  The
 * reference has no batch layer: each sonicSolver run is one case; a batch is
 * the GPU form of running many cases (test/Sod-style cases, MPI ranks on
 * independent blocks) side by side.  Every grid can carry its own numerics
 * (recipe, gamma, CFL, maxDeltaT: sfg_batch_add_ex), as every reference case
 * directory selects its own TermRecipe; the time recipe and precision mode
 * are the batch's.  State memory comes from one slab of `hbm_budget_bytes`
 * reserved at create; sfg_batch_add returns SFG_ERR_BUDGET when a grid does
 * not fit. */
typedef struct sfg_batch_s* sfg_batch;
int sfg_batch_create(const sfg_numerics_desc* numerics, size_t hbm_budget_bytes, int max_instances,
                     void* stream, sfg_batch* out);
int sfg_batch_destroy(sfg_batch b);
/* Device bytes a grid would take from the budget. */
int sfg_batch_instance_bytes(sfg_batch b, const sfg_grid_desc* grid, size_t* bytes);
/* Uploads a grid (AoS nodes, time 0) that will run to t_end or max_steps
 * (<= 0: no step limit); *slot identifies it. */
int sfg_batch_add(sfg_batch b, const sfg_grid_desc* grid, const double* host_nodes_aos, double t_end,
                  int64_t max_steps, int* slot);
/* sfg_batch_add with the grid's own numerics (NULL: the batch's): any recipe
 * the batch kernels provide (WENO3/5/7, TENO5 x Rusanov/Roe) with its gamma,
 * CFL and maxDeltaT; time_recipe and precision must equal the batch's
 * (SFG_ERR_ARG otherwise).  Grids of one recipe share that recipe's stage
 * kernel; up to 8 recipes per batch.  The reference binds one TermRecipe per
 * case (core/config/types/SF_termRecipe.h:242-259): this is that choice, per
 * grid of a batch. */
int sfg_batch_add_ex(sfg_batch b, const sfg_grid_desc* grid, const sfg_numerics_desc* numerics,
                     const double* host_nodes_aos, double t_end, int64_t max_steps, int* slot);
/* sfg_batch_add_ex for a grid with boundary ends of every kind a single-grid
 * solver takes: frozen ends (SFG_BC_FROZEN: a patch without a condition)
 * and law ends (SFG_BC_LAW) whose laws are laws[2 * axis + end] (read only
 * at those ends; may be NULL when the grid has none), checked as
 * sfg_set_boundary_law checks them.  The laws run where the single-grid
 * solver runs them (the step's start, before every stage's RHS, after the
 * last stage) with the same arithmetic, so a grid gives the same results in
 * a batch as alone: a reference case with a fixedValue inflow, a noSlip wall
 * or an unconditioned patch (Boundary::Applicator, solver/boundary/
 * SF_applicator.h:51-83, 162-187) runs batched as written. */
int sfg_batch_add_laws(sfg_batch b, const sfg_grid_desc* grid, const sfg_numerics_desc* numerics,
                       const sfg_boundary_law* laws, const double* host_nodes_aos, double t_end, int64_t max_steps,
                       int* slot);
/* Output clipping of one grid, as sfg_advance's write_interval: its steps
 * stop exactly at every write_interval after its current time (<= 0:
 * none), so its dt sequence equals a single-grid run that writes output at
 * those times (Time::Driver, src/solver/algorithm/time/SF_time.cpp:56-72).
 * Call between steps. */
int sfg_batch_set_write_interval(sfg_batch b, int slot, double write_interval);
int sfg_batch_remove(sfg_batch b, int slot);
/* Runs up to `steps` batch steps (graph of `graph_steps`, <= 0: 16); stops
 * early when no grid is running.  *active = grids that stepped last. */
int sfg_batch_step(sfg_batch b, int steps, int graph_steps, int* active);
int sfg_batch_status(sfg_batch b, int slot, double* time, int64_t* steps, int* running, uint32_t* flags);
int sfg_batch_download(sfg_batch b, int slot, double* host_nodes_aos);
/* Tile shape of the 2-D work items: 1 = 32 x 15, 2 = 22 x 22. */
int sfg_batch_set_variant(sfg_batch b, int variant);
int sfg_batch_info(sfg_batch b, size_t* used_bytes, size_t* budget_bytes, int* live, int* items);
/* Status of slots 0..count-1 in one read (running: 1 running, 0 finished or
 * failed, -1 empty slot); any output pointer may be NULL. */
int sfg_batch_snapshot(sfg_batch b, int count, int* running, double* time, int64_t* steps, uint32_t* flags);

/* ---- serving -------------------------------------------------------------
 * A request loop on its own host thread over one batch: submitted solves
 * wait in a FIFO queue, are admitted while the HBM budget and the slot count
 * allow, step with everything else in flight (state stays on the device),
 * and are retired -- result downloaded, slot and memory released -- as soon
 * as they finish.  Requests arriving while others run join the batch at the
 * next graph boundary (continuous batching). */
enum { SFG_REQ_QUEUED = 0, SFG_REQ_RUNNING = 1, SFG_REQ_DONE = 2, SFG_REQ_FAILED = 3, SFG_REQ_CANCELLED = 4 };
typedef struct {
    double submit_s, admit_s, finish_s;  /* seconds on the server's steady clock */
    int64_t steps;
    double time;
    uint32_t flags;
    int state;                           /* SFG_REQ_* */
} sfg_request_info;
typedef struct sfg_server_s* sfg_server;
int sfg_server_create(const sfg_numerics_desc* numerics, size_t hbm_budget_bytes, int max_slots, int graph_steps,
                      sfg_server* out);
/* Stops the loop (pending requests are cancelled) and frees everything. */
int sfg_server_destroy(sfg_server s);
/* Copies the input; the request runs to t_end or max_steps. */
int sfg_server_submit(sfg_server s, const sfg_grid_desc* grid, const double* host_nodes_aos, double t_end,
                      int64_t max_steps, int64_t* request_id);
/* sfg_server_submit with the request's own numerics (NULL: the server's),
 * under the rules of sfg_batch_add_ex, checked before the request queues. */
int sfg_server_submit_ex(sfg_server s, const sfg_grid_desc* grid, const sfg_numerics_desc* numerics,
                         const double* host_nodes_aos, double t_end, int64_t max_steps, int64_t* request_id);
/* sfg_server_submit_ex with the grid's boundary laws (laws[2 * axis + end]
 * for its SFG_BC_LAW ends; NULL when it has none), under the rules of
 * sfg_batch_add_laws, checked before the request queues. */
int sfg_server_submit_laws(sfg_server s, const sfg_grid_desc* grid, const sfg_numerics_desc* numerics,
                           const sfg_boundary_law* laws, const double* host_nodes_aos, double t_end,
                           int64_t max_steps, int64_t* request_id);
int sfg_server_poll(sfg_server s, int64_t request_id, sfg_request_info* info);
/* Result of a finished request (AoS nodes); SFG_ERR_ARG while not done. */
int sfg_server_fetch(sfg_server s, int64_t request_id, double* host_nodes_aos);
int sfg_server_cancel(sfg_server s, int64_t request_id);
/* Blocks until every submitted request has left the system or timeout_s
 * passes (SFG_ERR_TIMEOUT). */
int sfg_server_drain(sfg_server s, double timeout_s);
/* Seconds on the server's steady clock (same origin as sfg_request_info). */
double sfg_server_now(sfg_server s);

/* Kernel variant of the stage operator: 0 = one sweep launch per axis
 * (any dimension), 1 = fused tile kernel (2-D: 32 x 15 tiles, 1-D: 511-node
 * tiles, 3-D: 16 x 15 columns marching up 32-plane chunks), 2 = fused 2-D
 * tile kernel with 22 x 22 tiles; for 1-D grids variant 2 runs sfg_advance
 * in one thread-block cluster that steps the whole run on device (FP64, up to
 * 8192 nodes, no boundary laws, not Lax-Wendroff; other 1-D grids and single
 * stages use the 1-D tiles).  sfg_create picks 2 for 1-D, 1 for 2-D and 0
 * for 3-D grids; results agree across variants to round-off (FP32-flux: every
 * face takes the stage's one reference state; the sweeps scale face fluxes
 * by the area in FP64, the tiles in FP32), and the tile variants give the
 * same bits as a batch. */
int sfg_set_kernel_variant(sfg_solver s, int variant);
int sfg_get_kernel_variant(sfg_solver s, int* variant);

/* ---- residual without device allocation --------------------------------
 * Has no counterpart in the reference.  Some callers cannot allocate device
 * memory where they need an operator evaluation: a host application whose
 * own memory manager owns the whole device budget and forbids plugins from
 * allocating, a deployment with a fixed, pre-sized memory plan, or code on a
 * latency-critical stream that must not take cudaMalloc's implicit device
 * synchronisation.  sfg_residual_noalloc computes the spatial residual
 * R = Jac * sum_d dF_d (0 on unsolved transmissive boundary nodes) of a
 * caller-owned device state and writes it to a caller-owned device array.
 * In FP64 it equals sfg_residual's to round-off; with SFG_PREC_FP32_FLUX it
 * runs the axis-sweep form, which scales each face flux by its area in FP64
 * where sfg_residual's tiles do it in FP32, so the two agree to FP32
 * round-off only.  It allocates nothing: its working memory is one fixed array in
 * the library's device image, of 32 + 5 * SFG_NOALLOC_MAX_NODES doubles
 * (~10 MiB), which every GPU that loads the library holds until the process
 * exits.
 *   dev_q, dev_r: device arrays, structure of arrays [5][nodes] with
 *                 nodes = n[0] * n[1] * n[2] (x fastest), FP64.
 *   stream:       cudaStream_t (NULL: the legacy default stream).
 * Grids of more than SFG_NOALLOC_MAX_NODES nodes are rejected (SFG_ERR_ARG).
 * The first call on each device looks up the array's device address with
 * that device current and keeps it for the life of the process; the entry
 * point is not valid across cudaDeviceReset.  Every call waits for its work
 * on `stream` and reads the status word back to the host, so it never runs
 * on a stream that is being captured (SFG_ERR_ARG).  All calls share the one
 * array and it keeps the last call's contents, so calls whose work overlaps
 * on the GPU (other streams, other host threads) race: serialise them. */
#define SFG_NOALLOC_MAX_NODES 262144
int sfg_residual_noalloc(const sfg_grid_desc* grid, const sfg_numerics_desc* numerics,
                         const double* dev_q, double* dev_r, void* stream);

/* ---- diagnostics (no counterpart in the reference: measurement aids) -- */
/* TENO5 cut-off decisions of the current state's faces (3 per scalar core,
 * 30 per face) evaluated in FP64 and in FP32: *flips counts those that
 * differ.  Zero for non-TENO recipes. */
int sfg_teno_flip_rate(sfg_solver s, uint64_t* decisions, uint64_t* flips);
/* Runs stage `stage` of a step of size dt `repeats` times on the current
 * state without committing it, timing each axis sweep with CUDA events on the
 * solver's stream; ms_per_axis[d] receives the mean duration of sweep d.  A
 * fused stage (tile kernels, curvilinear launches) is timed as `repeats`
 * launches captured in one CUDA graph, as it runs inside a step's graph
 * (ms_per_axis[0]; launch by launch on the legacy default stream). */
int sfg_time_sweeps(sfg_solver s, int stage, double dt, int repeats, float* ms_per_axis);
/* Dependent-FMA throughput of this GPU in TFLOP/s (fp64 = 1: double,
 * 0: float), measured with a kernel of `seconds` length. */
int sfg_measure_fma_peak(int fp64, double seconds, double* tflops);

#ifdef __cplusplus
}
#endif
#endif
