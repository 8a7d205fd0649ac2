/*
 * sf_oracle.h -- CPU oracle for the density-based explicit Euler path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * CPU algorithm (sonicSolver) used as the checker for the CUDA path.  Only
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
 * legs may load it.  The product library never links or calls it.
 *
 * Grid model (node based, as the reference Field, SF_field.h:26-67):
 *   - `dim` active axes are the first `dim` of (x, y, z);
 *   - n[d] nodes per axis (1 on inactive axes);
 *   - `ng` ghost layers on both sides of every active axis only;
 *   - state Q is AoS [k][j][i][v], v = (rho, rho u, rho v, rho w, E).
 * Storage extents are m[d] = n[d] + 2 ng on active axes, n[d] otherwise.
 */
#ifndef SF_ORACLE_H
#define SF_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Convection schemes, in the order of FDM::ConvectionScheme
 * (src/core/config/types/SF_termRecipe.h:14). */
enum { SFO_WENO3 = 0, SFO_WENO5 = 1, SFO_TENO5 = 2, SFO_WENO7 = 3 };
/* Face fluxes, in the order of FDM::FluxSplitter (SF_termRecipe.h:33-40). */
enum { SFO_STEGER = 0, SFO_RUSANOV = 1, SFO_LAXFRIEDRICHS = 2, SFO_ROE = 3,
       SFO_LAXWENDROFF = 4 };
/* Time recipes, in the order of FDM::TimeRecipeId (SF_timeRecipe.h:11). */
enum { SFO_EULER = 0, SFO_SSPRK3 = 1, SFO_RK4 = 2 };
/* Boundary kinds per axis end.
 *   TRANSMISSIVE: zeroGradient; the boundary node copies its inner neighbour
 *                 and is not advanced; ghosts copy the boundary node
 *                 (SF_zeroGradient.cpp:88-105, SF_iteration.h:36-46).
 *   PERIODIC:     ghosts wrap; every node is advanced (no reference code).
 *   FROZEN:       no boundary law: the boundary node is advanced and the
 *                 ghosts keep the values they were given (SF_applicator.h:162-187
 *                 with no BC configured for the set).
 *   LAW:          the reference's physical boundary laws per field
 *                 (Boundary::Applicator::apply, SF_applicator.h:51-83): a
 *                 density law, a velocity law and a pressure law (energy
 *                 rebuilt from pressure), each fixedValue, zeroGradient or
 *                 symmetry.  The boundary node is written by the laws and not
 *                 advanced; every ghost layer is derived from it. */
enum { SFO_BC_TRANSMISSIVE = 0, SFO_BC_PERIODIC = 1, SFO_BC_FROZEN = 2, SFO_BC_LAW = 3 };

/* Field laws of one LAW end (FDM::BoundaryConfig density / velocity /
 * pressure settings of one patch; BCSetting types FIXED_VALUE,
 * ZERO_GRADIENT, SYMMETRY). */
enum { SFO_LAW_ZERO_GRADIENT = 0, SFO_LAW_FIXED_VALUE = 1, SFO_LAW_SYMMETRY = 2 };
typedef struct {
    int rho, U, p;        /* SFO_LAW_* of density, velocity, pressure */
    int pad;
    double rho_value;     /* fixedValue density */
    double U_value[3];    /* fixedValue velocity */
    double p_value;       /* fixedValue pressure */
} sfo_law;

/* Error codes (the reference exits the process on these conditions). */
enum {
    SFO_OK = 0,
    SFO_ERR_NONFINITE = 1,     /* non-finite stencil / flux / state */
    SFO_ERR_STATE = 2,         /* rho <= 0 or p <= 0 */
    SFO_ERR_TENO_CUTOFF = 3,   /* TENO5 rejected all sub-stencils */
    SFO_ERR_ARG = 4,           /* invalid argument */
    SFO_ERR_ROE_SOUND = 5      /* Roe-averaged a^2 <= 0 */
};

typedef struct {
    int dim;            /* active axes: 1, 2 or 3 */
    int n[3];           /* nodes per axis */
    int ng;             /* ghost layers on active axes */
    double h[3];        /* node spacing (inactive axes: slab thickness) */
    int bc_lo[3];
    int bc_hi[3];
    double gamma;
    const sfo_law* law;  /* law[2 * axis + end] of SFO_BC_LAW ends (end 0 = low) */
    /* Curvilinear grids: 10 doubles per storage point of Q's layout (ghosts
     * included): Jac (= 1/J), XiX, XiY, XiZ, EtX, EtY, EtZ, ZeX, ZeY, ZeZ, as
     * the reference Field holds them.  NULL: uniform Cartesian metrics from h. */
    const double* metrics;
} sfo_grid;

/* Counters reported by the oracle (TENO cut-off decisions etc.). */
typedef struct {
    unsigned long long teno_cores;      /* TENO5 core evaluations */
    unsigned long long teno_cut;        /* sub-stencils cut (chi_k = 0) */
    unsigned long long faces;           /* faces evaluated */
} sfo_counters;

long long sfo_storage_size(const sfo_grid* g);   /* doubles in Q */

/* Scalar cores (exposed for known-answer tests). */
double sfo_weno3_core(const double* v);
double sfo_weno5_core(const double* v);
double sfo_weno7_core(const double* v);
double sfo_teno5_core(const double* v, int* cut_mask);

/* L and R (row-major 5x5) at q for unit normal n; returns error code. */
int sfo_char_matrix(const double* q, const double* n, double gamma,
                    double* L, double* R);
/* Face fluxes (no area factor). */
int sfo_rusanov_flux(const double* qL, const double* qR, const double* n,
                     double gamma, double* out);
int sfo_roe_flux(const double* qL, const double* qR, const double* n,
                 double gamma, double* out);
int sfo_steger_flux(const double* qL, const double* qR, const double* n,
                    double gamma, double* out);
int sfo_lf_flux(const double* qL, const double* qR, const double* n,
                double gamma, double* out);
/* Lax-Wendroff needs the step size and the face spacing (both > 0). */
int sfo_lw_flux(const double* qL, const double* qR, const double* n, double dt,
                double spacing, double gamma, double* out);
/* One characteristic face flux from a (2r)-point conservative stencil
 * (nstencil = 4, 6, 8) and the face metrics [sx, sy, sz, 1/J]; result is
 * multiplied by the face area (SF_WENO.h:184-245). */
int sfo_char_face_flux(int nstencil, const double* stencil, const double* metrics,
                       int scheme, int flux, double gamma, double* out);
/* The same with the Lax-Wendroff step size and face spacing. */
int sfo_char_face_flux_ex(int nstencil, const double* stencil, const double* metrics,
                          int scheme, int flux, double gamma, double dt, double spacing,
                          double* out);
/* Step size the Lax-Wendroff flux of sfo_rhs uses (set by the stage
 * functions from their dt; sfo_rhs alone needs it set explicitly). */
void sfo_set_step_dt(double dt);
double sfo_step_dt(void);

/* Apply the boundary laws of g to the ghost layers / boundary nodes of Q. */
int sfo_fill_ghosts(const sfo_grid* g, double* Q);
/* Spatial residual R = Jac * sum_d (F_d[i] - F_d[i-1]) at every interior
 * node (R has the same layout as Q; ghost entries are set to 0). */
int sfo_rhs(const sfo_grid* g, int scheme, int flux, const double* Q, double* R,
            sfo_counters* counters);
/* CFL time step over the solved nodes (SF_rusanovEOS.cpp:110-147). */
int sfo_dt(const sfo_grid* g, const double* Q, double cfl, double* dt);
/* One explicit step of size dt: ghost fill before every stage, stage
 * combination on solved nodes, ghost fill after the step (commit).
 * `work` must hold 5 * sfo_storage_size(g) doubles. */
int sfo_step(const sfo_grid* g, int scheme, int flux, int time_id, double* Q,
             double dt, double* work, sfo_counters* counters);
/* One stage of a step (for stage-granularity parity): `stage` in
 * [0, stages); q0/k1..k4 live in `work` as for sfo_step. stage 0 snapshots
 * q0.  After the last stage the commit ghost fill is applied. */
int sfo_stage(const sfo_grid* g, int scheme, int flux, int time_id, double* Q,
              double dt, int stage, double* work, sfo_counters* counters);
/* Time loop of Time::Driver::run (SF_time.cpp:42-93): dt = min(CFL dt,
 * max_dt, remaining, next output time - t).  Records each dt in dt_out
 * (capacity max_steps).  Returns error code; *steps_done, *t_final set. */
int sfo_advance(const sfo_grid* g, int scheme, int flux, int time_id, double* Q,
                double t_start, double t_end, double cfl, double max_dt,
                double write_interval, int max_steps, double* dt_out,
                int* steps_done, double* t_final, sfo_counters* counters);

/* The same stage / time loops around a caller-supplied spatial operator and
 * CFL routine (used to run the reference's own operator in oracle/_ref). */
typedef int (*sfo_rhs_fn)(void* ctx, const double* Q, double* R);
typedef int (*sfo_dt_fn)(void* ctx, const double* Q, double cfl, double* dt);
int sfo_stage_fn(const sfo_grid* g, sfo_rhs_fn rhs, void* ctx, int time_id, double* Q, double dt,
                 int stage, double* work);
int sfo_advance_fn(const sfo_grid* g, sfo_rhs_fn rhs, sfo_dt_fn dtf, void* ctx, int time_id,
                   double* Q, double t_start, double t_end, double cfl, double max_dt,
                   double write_interval, int max_steps, double* dt_out, int* steps_done,
                   double* t_final);

#ifdef __cplusplus
}
#endif
#endif
