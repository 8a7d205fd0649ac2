// sfg_internal.h -- structures shared by the host runtime and the kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/sonicsolver_b200.h"

namespace sfg {

constexpr int BC_TRANSMISSIVE = 0;
constexpr int BC_PERIODIC = 1;
// A frozen end: the device grid carries one extra, never advanced node at
// that end holding the frozen ghost value, and ghost indices clamp to it.
constexpr int BC_FROZEN = 2;

// Status bits (match SFG_FLAG_* in include/sonicsolver_b200.h).
constexpr unsigned FLAG_NONFINITE = 1u << 0;
constexpr unsigned FLAG_DENSITY = 1u << 1;
constexpr unsigned FLAG_PRESSURE = 1u << 2;
constexpr unsigned FLAG_TENO_CUTOFF = 1u << 3;
constexpr unsigned FLAG_ROE_SOUND = 1u << 4;

// Reconstruction schemes in the order of FDM::ConvectionScheme and face
// fluxes with the values of FDM::FluxSplitter (SF_termRecipe.h:14,33-40).
enum Scheme { WENO3 = 0, WENO5 = 1, TENO5 = 2, WENO7 = 3 };
enum Flux { STEGER = 0, RUSANOV = 1, LAXF = 2, ROE = 3, LAXW = 4 };

// Device-resident step clock: the Time::Driver bookkeeping
// (src/solver/algorithm/time/SF_time.cpp:42-93) and FlowDtCompute's
// min(dt, maxDeltaT, limit) (SF_flowOperations.cpp:487-513) kept on the GPU so
// that whole runs of steps execute inside one CUDA graph.
struct Clock {
    double t;                 // physical time
    double t_end;             // run end (inf: none)
    double next_out;          // next output time (inf: none)
    double write_interval;    // <= 0: none
    double max_dt;            // numerics maxDeltaT (inf: none)
    double limit;             // one-shot extra limit (inf: none)
    double dt;                // step size of the current step
    unsigned long long dt_bits;  // CFL minimum, as ordered bits of a positive double
    long long steps;
    long long max_steps;
    long long log_base;       // step index of dt_log[0]
    int active;               // 1 while the current step runs
    int dt_ready;             // 1: dt_bits already holds the CFL minimum of the current
                              // state (reduced by the previous step's last stage)
};

// Geometry of one grid as the kernels see it (uniform Cartesian metrics).
struct GridView {
    int n[3];          // nodes per axis (1 on inactive axes)
    int lo[3], hi[3];  // solved node range per axis
    int bc_lo[3], bc_hi[3];
    int dim;
    long long vs;      // distance between variables in the SoA state (doubles)
    double jac;        // 1 / J
    double area[3];    // face cofactor magnitude per axis
    double metric[3];  // xi_x, eta_y, zeta_z
    double gamma;
    double cfl;
    double h[3];       // node spacing (the Lax-Wendroff face spacing)
    // Curvilinear grids (curv = 1; sfg_set_metrics): per-node metrics and
    // per-face geometry replace jac / area / metric.
    int curv;
    const double* node_jac;     // Jac = 1/J per node (vs doubles)
    const double* node_metric;  // xi_x, xi_y, xi_z, eta_x, ..., zeta_z per node (9 x vs)
    const double* geom[3];      // per axis, face (i | i+1) at its lower node i: unit normal, area (4 x vs)
};

// Physical boundary laws of the law ends of one grid (SFG_BC_LAW; the
// kernels see such an end as BC_FROZEN: one extra node holding the ghost
// value, the boundary node outside the solved range).
constexpr int LAW_ZERO_GRADIENT = 0, LAW_FIXED_VALUE = 1, LAW_SYMMETRY = 2;
struct LawView {
    int count;              // law ends
    int axis[6], end[6];
    int rho[6], U[6], p[6]; // LAW_* per field
    double rho_value[6], U_value[6][3], p_value[6];
    long long start[7];     // prefix sums of the face points per law end
    // per face point: which state of its boundary node the pressure law reads
    // (LAW_STATE_*), as the reference's state cache hands it out
    const unsigned char* codes;
};
constexpr int LAW_STATE_FRESH = 0;   // the boundary node's new state
constexpr int LAW_STATE_PRIMED = 1;  // new density, momentum and energy before the application
constexpr int LAW_STATE_HALF = 2;    // new density and momentum, energy before the application

// Stage arithmetic of one launch (Time::Explicit, SF_explicit.cpp:193-238,282-285).
enum TimeId { T_EULER = 0, T_SSPRK3 = 1, T_RK4 = 2 };

struct StageView {
    const double* qs;     // state read by the stencils (current stage input)
    const double* q0;     // step-start state
    double* qout;         // stage output
    double* r;            // residual accumulator (SoA)
    double* k;            // RK4 accumulator (SoA)
    Clock* clock;
    unsigned* flags;
    unsigned long long* counters;  // [teno cores, teno cut] or null
    int time_id;
    int stage;
    double base, inc;     // SSPRK3: base*q0 + inc*(q - dt R);  RK4: inc = stage weight
    int mode;             // MODE_* bits
    int require_active;   // skip when clock->active == 0
};

constexpr int MODE_READ_R = 1;     // add the residual accumulated by earlier axes
constexpr int MODE_FINAL = 2;      // last axis: finish the node
constexpr int MODE_RESIDUAL = 4;   // final output is R = Jac * div (no stage update)
constexpr int MODE_CFL = 8;        // last stage of a step: also reduce the CFL minimum of
                                   // the new state into clock->dt_bits (the next step's dt)

// One launch of the 1-D whole-run cluster kernel (sfg_cluster1d.cu): the
// stage views of a step, the clock it advances and where it logs.
struct ClusterRun {
    StageView sv[4];         // the step's stages: recipe and coefficients; sv[0].qs is qn,
                             // loaded at the start and stored at the end (the stage
                             // buffers themselves live in the cluster's shared memory)
    int stages;
    Clock* clock;
    double* dt_log;
    long long dt_cap;
    unsigned* flags;
    long long launch_steps;  // steps per launch at most (the host relaunches)
};

// Host helpers of the boundary laws (sfg_runtime.cu): the checks of one
// end's laws (nullptr: valid), and the law view plus the reference
// state-cache replay codes of a grid that is not a solver of its own.
const char* law_problem(const sfg_boundary_law& law);
void grid_law_view(const sfg_grid_desc& G, const GridView& gv, const int off_lo[3], const sfg_boundary_law* laws,
                   int ng, LawView& lv, std::vector<unsigned char>& codes);

// A named NVTX range over a host scope: the C-ABI entries mark their work
// for a timeline profiler (Nsight Systems) and for range filters (ncu
// --nvtx-include).  Without a tool attached a push / pop costs a branch.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

// One-time kernel attribute setup per device: kernel attributes belong to a
// device context, so each launcher keeps its own set of devices done (one bit
// per device ordinal).  Sets `bit` to the current device's bit.
inline bool attributes_pending(const std::atomic<unsigned long long>& done, unsigned long long& bit) {
    int dev = 0;
    cudaGetDevice(&dev);
    bit = 1ull << (dev & 63);
    return !(done.load(std::memory_order_acquire) & bit);
}

}  // namespace sfg
