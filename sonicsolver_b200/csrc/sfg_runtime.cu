// sfg_runtime.cu -- host runtime behind the C ABI (include/sonicsolver_b200.h).
//
// A solver handle owns the device state of one grid, a stream, the
// device-resident step clock and, for sfg_advance, a CUDA graph of a run of
// steps.  This is the B200-native counterpart of what FlowOperations binds for
// the flow.conservative provider (src/solver/algorithm/SF_flowOperations.cpp:466-522):
// FlowStepPrepare (ghost fill -> index mapping in the kernels), FlowDtCompute
// (dt_kernel + finalize), FlowStepBegin (q0 is the untouched step-start
// buffer), ExplicitStageExecute (sweep launches), FlowStepCommit / TimeCommit
// (commit_kernel).
#include "../../include/sonicsolver_b200.h"
#include "sfg_internal.h"

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <limits>
#include <string>
#include <unordered_set>
#include <vector>

namespace sfg {
cudaError_t launch_sweep(int scheme, int flux, int prec64, int axis, const GridView& g, const StageView& sv,
                         cudaStream_t st);
cudaError_t launch_dt(const GridView& g, const double* q, Clock* clock, unsigned* flags, int skip_if_ready,
                      cudaStream_t st);
cudaError_t launch_finalize_dt(Clock* c, const unsigned* flags, cudaStream_t st);
cudaError_t launch_commit(Clock* c, double* dt_log, long long dt_cap, int cfl_next, cudaStream_t st);
cudaError_t launch_set_dt(Clock* c, double dt, cudaStream_t st);
cudaError_t launch_reset_min(Clock* c, cudaStream_t st);
cudaError_t launch_stage_from_residual(const GridView& g, const StageView& sv, cudaStream_t st);
cudaError_t launch_aos_to_soa(const double* aos, double* soa, long long nodes, long long vs, cudaStream_t st);
cudaError_t launch_soa_to_aos(const GridView& g, const double* soa, double* aos, cudaStream_t st);
cudaError_t launch_totals(const GridView& g, const double* q, double* out, double vol, cudaStream_t st);
cudaError_t launch_tile2d(int variant, int scheme, int flux, int prec64, const GridView& g, const StageView& sv,
                          cudaStream_t st);
cudaError_t launch_tile1d(int scheme, int flux, int prec64, const GridView& g, const StageView& sv, cudaStream_t st);
cudaError_t launch_tile3d(int scheme, int flux, int prec64, const GridView& g, const StageView& sv, cudaStream_t st);
cudaError_t launch_law_fill(const GridView& g, const LawView& lv, const double* old, double* q, const Clock* clock,
                            int require_active, unsigned* flags, cudaStream_t st);
cudaError_t launch_curv_geometry(const GridView& g, const double* nm, double* const geom[3], unsigned* flags,
                                 cudaStream_t st);
cudaError_t launch_curv_stage(int scheme, int flux, int prec64, int tiles, const GridView& g, const StageView& sv,
                              double* fl, cudaStream_t st);
cudaError_t launch_teno_flips(const GridView& g, const double* q, unsigned long long* out, cudaStream_t st);
bool cluster1d_eligible(const GridView& g, int flux, int prec64);
cudaError_t launch_cluster1d(int scheme, int flux, const GridView& g, const ClusterRun& run, cudaStream_t st);
}  // namespace sfg

using namespace sfg;

namespace {

thread_local std::string g_error;

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_error = buf;
    return code;
}

#define CUDA_TRY(expr)                                                                          \
    do {                                                                                        \
        cudaError_t e_ = (expr);                                                                \
        if (e_ != cudaSuccess) return fail(SFG_ERR_CUDA, "%s: %s", #expr, cudaGetErrorString(e_)); \
    } while (0)

struct RecipeInfo {
    int id;
    const char* name;
    int scheme;  // sfg::Scheme
    int flux;    // sfg::Flux
};

// The convection recipes of FDM::TermRecipeId served here (names of
// FDM::toString(TermRecipeId), SF_termRecipe.h:242-259).
const RecipeInfo kRecipes[] = {
    {SFG_RECIPE_WENO3_RUSANOV, "weno3Rusanov", WENO3, RUSANOV},
    {SFG_RECIPE_WENO3_ROE, "weno3Roe", WENO3, ROE},
    {SFG_RECIPE_WENO5_RUSANOV, "weno5Rusanov", WENO5, RUSANOV},
    {SFG_RECIPE_WENO5_ROE, "weno5Roe", WENO5, ROE},
    {SFG_RECIPE_TENO5_RUSANOV, "teno5Rusanov", TENO5, RUSANOV},
    {SFG_RECIPE_TENO5_ROE, "teno5Roe", TENO5, ROE},
    {SFG_RECIPE_WENO7_RUSANOV, "weno7Rusanov", WENO7, RUSANOV},
    {SFG_RECIPE_WENO7_ROE, "weno7Roe", WENO7, ROE},
    {SFG_RECIPE_WENO3_STEGER, "weno3Steger", WENO3, STEGER},
    {SFG_RECIPE_WENO3_LAXF, "weno3LaxFriedrichs", WENO3, LAXF},
    {SFG_RECIPE_WENO3_LAXW, "weno3LaxWendroff", WENO3, LAXW},
    {SFG_RECIPE_WENO5_STEGER, "weno5Steger", WENO5, STEGER},
    {SFG_RECIPE_WENO5_LAXF, "weno5LaxFriedrichs", WENO5, LAXF},
    {SFG_RECIPE_WENO5_LAXW, "weno5LaxWendroff", WENO5, LAXW},
    {SFG_RECIPE_TENO5_STEGER, "teno5Steger", TENO5, STEGER},
    {SFG_RECIPE_TENO5_LAXF, "teno5LaxFriedrichs", TENO5, LAXF},
    {SFG_RECIPE_TENO5_LAXW, "teno5LaxWendroff", TENO5, LAXW},
    {SFG_RECIPE_WENO7_STEGER, "weno7Steger", WENO7, STEGER},
    {SFG_RECIPE_WENO7_LAXF, "weno7LaxFriedrichs", WENO7, LAXF},
    {SFG_RECIPE_WENO7_LAXW, "weno7LaxWendroff", WENO7, LAXW},
};

const RecipeInfo* find_recipe(int id) {
    for (const auto& r : kRecipes)
        if (r.id == id) return &r;
    return nullptr;
}

int ghost_layers(int scheme) { return scheme == WENO3 ? 2 : (scheme == WENO7 ? 4 : 3); }
int stage_count(int time_id) { return time_id == T_EULER ? 1 : (time_id == T_SSPRK3 ? 3 : 4); }

}  // namespace

namespace sfg {
// Records a failure message for sfg_last_error() from other translation units.
void set_last_error(const char* msg) { g_error = msg ? msg : ""; }
}  // namespace sfg

struct sfg_solver_s {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    sfg_grid_desc grid{};  // as the caller described it
    // Device grid: `grid` plus one extra node at every frozen end, which
    // holds the frozen ghost value and is never advanced.
    sfg_grid_desc ig{};
    int off_lo[3] = {0, 0, 0};  // 1 where the low end is frozen or a law end
    bool frozen = false;        // the device grid has extra nodes (frozen or law ends)
    bool has_laws = false;      // some end is SFG_BC_LAW
    sfg_boundary_law laws[6] = {};  // [2 * axis + end]
    LawView lv{};
    unsigned char* law_codes = nullptr;  // device: LAW_STATE_* per law face point
    // curvilinear grids (sfg_set_metrics)
    double* node_metrics = nullptr;  // Jac then the 9 metric components per node (10 x vs)
    double* face_geom = nullptr;     // unit normal and area per face, per axis (3 x 4 x vs)
    double* face_flux = nullptr;     // face fluxes of one stage, per axis (3 x 5 x vs)
    long long pub_nodes = 0;    // nodes of `grid`
    sfg_numerics_desc num{};
    const RecipeInfo* recipe = nullptr;
    int ng = 3;
    GridView gv{};
    long long nodes = 0;        // nodes of the device grid
    double *qn = nullptr, *qa = nullptr, *qb = nullptr, *r = nullptr, *k = nullptr, *staging = nullptr;
    double* totals = nullptr;
    Clock* clock = nullptr;
    unsigned* flags = nullptr;
    unsigned long long* counters = nullptr;
    bool counting = false;
    int variant = 0;  // stage-operator kernel variant (sfg_set_kernel_variant)
    int next_stage = 0;
    double stage_dt = 0.0;
    // graph of `graph_steps` steps for sfg_advance
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0;
    double* dt_log = nullptr;
    long long dt_log_cap = 0;
    Clock* host_clock = nullptr;  // pinned mirror
};

namespace {

int validate(const sfg_grid_desc* g, const sfg_numerics_desc* n, const RecipeInfo** recipe) {
    if (!g || !n) return fail(SFG_ERR_ARG, "null descriptor");
    if (g->dim < 1 || g->dim > 3) return fail(SFG_ERR_ARG, "dim must be 1..3 (got %d)", g->dim);
    const RecipeInfo* r = find_recipe(n->recipe);
    if (!r) return fail(SFG_ERR_ARG, "convection recipe %d is not provided on the GPU", n->recipe);
    if (n->time_recipe < 0 || n->time_recipe > 2) return fail(SFG_ERR_ARG, "unknown time recipe %d", n->time_recipe);
    if (n->precision != SFG_PREC_FP64 && n->precision != SFG_PREC_FP32_FLUX)
        return fail(SFG_ERR_ARG, "unknown precision mode %d", n->precision);
    if (n->precision == SFG_PREC_FP32_FLUX && r->flux != RUSANOV && r->flux != ROE)
        return fail(SFG_ERR_ARG, "%s: the FP32-flux mode implements Rusanov and Roe faces (use FP64)", r->name);
    if (!(n->gamma > 1.0) || !std::isfinite(n->gamma)) return fail(SFG_ERR_ARG, "gamma must be > 1");
    if (!(n->cfl > 0.0) || !std::isfinite(n->cfl)) return fail(SFG_ERR_ARG, "CFL must be finite and > 0");
    const int reach = r->scheme == WENO3 ? 2 : (r->scheme == WENO7 ? 4 : 3);
    for (int d = 0; d < 3; ++d) {
        if (!(g->h[d] > 0.0) || !std::isfinite(g->h[d])) return fail(SFG_ERR_ARG, "h[%d] must be > 0", d);
        if (d >= g->dim) {
            if (g->n[d] != 1) return fail(SFG_ERR_ARG, "inactive axis %d must have 1 node", d);
            continue;
        }
        const bool plo = g->bc_lo[d] == SFG_BC_PERIODIC, phi = g->bc_hi[d] == SFG_BC_PERIODIC;
        if (plo != phi) return fail(SFG_ERR_ARG, "axis %d: periodic must be set on both ends", d);
        for (int b : {g->bc_lo[d], g->bc_hi[d]})
            if (b != SFG_BC_TRANSMISSIVE && b != SFG_BC_PERIODIC && b != SFG_BC_FROZEN && b != SFG_BC_LAW)
                return fail(SFG_ERR_ARG, "axis %d: unknown boundary kind %d", d, b);
        if ((g->bc_lo[d] == SFG_BC_LAW || g->bc_hi[d] == SFG_BC_LAW) && g->n[d] < 3)
            return fail(SFG_ERR_ARG, "axis %d: a law end needs >= 3 nodes", d);
        if (plo && g->n[d] < reach + 1) return fail(SFG_ERR_ARG, "periodic axis %d needs >= %d nodes", d, reach + 1);
        const int extra = (g->bc_lo[d] == SFG_BC_FROZEN || g->bc_lo[d] == SFG_BC_LAW) +
                          (g->bc_hi[d] == SFG_BC_FROZEN || g->bc_hi[d] == SFG_BC_LAW);
        if (!plo && g->n[d] + extra < 3) return fail(SFG_ERR_ARG, "axis %d needs >= %d nodes", d, 3 - extra);
    }
    *recipe = r;
    return SFG_OK;
}

// The reference reads the boundary node's state for a pressure law through
// the Field's thermodynamic state cache (Field::thermodynamicState,
// SF_field.cpp:133-151; ThermodynamicStateCache: min(storage points, 4096)
// direct-mapped entries keyed by the Field cell index, emptied before each
// application of the laws).  Which state a point's pressure law gets depends
// only on the grid and the laws, so this replays the sequence of cache
// queries of one application -- velocity laws of every law end, then
// pressure laws, face points with the last axis outermost, corners included
// (SF_fixedValue.cpp:129-160, SF_thermodynamicClosure.cpp:219-285) -- and
// records LAW_STATE_* for each face point the kernel updates.
void simulate_law_cache(const LawView& lv, const sfg_grid_desc& G, const GridView& gv, const int off_lo[3], int ng,
                        std::vector<unsigned char>& codes) {
    const long long mx = G.n[0] + 2LL * ng, my = G.n[1] + 2LL * ng, mz = G.n[2] + 2LL * ng;
    const long long cap = std::min<long long>(mx * my * mz, 4096);
    std::vector<long long> slot_cell((size_t)cap, -1);
    std::vector<unsigned char> slot_kind((size_t)cap, 0);
    codes.assign((size_t)lv.start[lv.count], (unsigned char)LAW_STATE_FRESH);
    auto cell = [&](const int (&p)[3]) {
        return ((long long)(p[2] + ng) * my + (p[1] + ng)) * mx + (p[0] + ng);
    };
    auto query = [&](long long c, unsigned char kind_if_miss) {
        const size_t sl = (size_t)(c % cap);
        if (slot_cell[sl] == c) return slot_kind[sl];
        slot_cell[sl] = c;
        slot_kind[sl] = kind_if_miss;
        return kind_if_miss;
    };
    int pub_lo[3], pub_hi[3];
    for (int d = 0; d < 3; ++d) {
        pub_lo[d] = gv.lo[d] - off_lo[d];
        pub_hi[d] = gv.hi[d] - off_lo[d];
    }
    // Boundary nodes whose energy this application has not written yet: an
    // edge point's inner sample can be another end's boundary node, and the
    // state cached for it then (new density and momentum, old energy) is the
    // one that end's pressure law finds.
    std::unordered_set<long long> pending;
    for (int e = 0; e < lv.count; ++e) {
        const int a = lv.axis[e], bnode = lv.end[e] ? G.n[a] - 1 : 0;
        int p[3];
        for (p[2] = 0; p[2] < G.n[2]; ++p[2])
            for (p[1] = 0; p[1] < G.n[1]; ++p[1])
                for (p[0] = 0; p[0] < G.n[0]; ++p[0])
                    if (p[a] == bnode) pending.insert(cell(p));
    }
    for (int family = 1; family <= 2; ++family)   // density laws query nothing
        for (int e = 0; e < lv.count; ++e) {
            const int a = lv.axis[e], hi = lv.end[e], n = G.n[a];
            if (family == 1 && lv.U[e] != LAW_FIXED_VALUE) continue;
            int p[3];
            for (p[2] = 0; p[2] < G.n[2]; ++p[2])
                for (p[1] = 0; p[1] < G.n[1]; ++p[1])
                    for (p[0] = 0; p[0] < G.n[0]; ++p[0]) {
                        if (p[a] != (hi ? n - 1 : 0)) continue;
                        const long long cb = cell(p);
                        int q[3] = {p[0], p[1], p[2]};
                        if (family == 1) {
                            query(cb, LAW_STATE_PRIMED);              // setMomentumFromVelocity(b)
                            for (int k = 0; k < ng; ++k) {
                                query(cb, LAW_STATE_HALF);            // primitiveVelocity(b)
                                q[a] = hi ? n + k : k - ng;
                                query(cell(q), 3);                    // setMomentumFromVelocity(ghost)
                            }
                            continue;
                        }
                        if (lv.p[e] != LAW_FIXED_VALUE) {
                            q[a] = hi ? n - 2 : 1;
                            const long long cs = cell(q);               // pressureAt(inner sample)
                            query(cs, pending.count(cs) ? LAW_STATE_HALF : LAW_STATE_FRESH);
                        }
                        pending.erase(cb);                              // setEnergyFromPressure(b)
                        unsigned char kind = query(cb, LAW_STATE_FRESH);  // pressureAt(b), every layer alike
                        bool face = true;
                        long long at = 0, mult = 1;
                        for (int d = 0; d < 3; ++d) {
                            if (d == a) continue;
                            face &= p[d] >= pub_lo[d] && p[d] < pub_hi[d];
                            at += (long long)(p[d] - pub_lo[d]) * mult;
                            mult *= pub_hi[d] - pub_lo[d];
                        }
                        if (face) codes[(size_t)(lv.start[e] + at)] = kind > LAW_STATE_HALF ? LAW_STATE_FRESH : kind;
                    }
        }
}

// Law ends of a grid (`G`, caller layout; `g`, its device view) in the order
// x low, x high, y low, ...; face points over the solved range of the other
// axes; laws[2 axis + end] holds each end's laws.
void make_law_view(const sfg_grid_desc& G, const GridView& g, const sfg_boundary_law* laws, LawView& lv) {
    lv = LawView{};
    for (int a = 0; a < G.dim; ++a)
        for (int end = 0; end < 2; ++end) {
            if ((end ? G.bc_hi[a] : G.bc_lo[a]) != SFG_BC_LAW) continue;
            const int e = lv.count++;
            const sfg_boundary_law& law = laws[2 * a + end];
            lv.axis[e] = a;
            lv.end[e] = end;
            lv.rho[e] = law.rho;
            lv.U[e] = law.velocity;
            lv.p[e] = law.pressure;
            lv.rho_value[e] = law.rho_value;
            for (int d = 0; d < 3; ++d) lv.U_value[e][d] = law.velocity_value[d];
            lv.p_value[e] = law.pressure_value;
            long long pts = 1;
            for (int d = 0; d < 3; ++d)
                if (d != a) pts *= g.hi[d] - g.lo[d];
            lv.start[e + 1] = lv.start[e] + pts;
        }
}

void build_law_view(sfg_solver_s* s) {
    make_law_view(s->grid, s->gv, s->laws, s->lv);
    s->lv.codes = s->law_codes;
}

// Device copy of the cache replay for the current laws (the number of face
// points never changes, so the buffer is allocated once).
int upload_law_codes(sfg_solver_s* s) {
    if (!s->lv.count) return SFG_OK;
    std::vector<unsigned char> codes;
    simulate_law_cache(s->lv, s->grid, s->gv, s->off_lo, s->ng, codes);
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    if (!s->law_codes && cudaMalloc((void**)&s->law_codes, codes.size()) != cudaSuccess) {
        s->law_codes = nullptr;
        return fail(SFG_ERR_NOMEM, "device allocation of the law table failed");
    }
    // on the solver's stream (non-blocking: the legacy stream does not order
    // against it), complete before `codes` goes out of scope
    CUDA_TRY(cudaMemcpyAsync(s->law_codes, codes.data(), codes.size(), cudaMemcpyHostToDevice, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    s->lv.codes = s->law_codes;
    return SFG_OK;
}

void make_view(sfg_solver_s* s) {
    // device grid: one extra node per frozen or law end
    s->ig = s->grid;
    s->frozen = false;
    s->has_laws = false;
    s->pub_nodes = (long long)s->grid.n[0] * s->grid.n[1] * s->grid.n[2];
    auto extra_end = [](int b) { return b == SFG_BC_FROZEN || b == SFG_BC_LAW; };
    for (int a = 0; a < s->grid.dim; ++a) {
        s->off_lo[a] = extra_end(s->grid.bc_lo[a]) ? 1 : 0;
        s->ig.n[a] += s->off_lo[a] + (extra_end(s->grid.bc_hi[a]) ? 1 : 0);
        s->frozen |= s->ig.n[a] != s->grid.n[a];
        s->has_laws |= s->grid.bc_lo[a] == SFG_BC_LAW || s->grid.bc_hi[a] == SFG_BC_LAW;
    }
    GridView& g = s->gv;
    const sfg_grid_desc& d = s->ig;
    g.dim = d.dim;
    for (int a = 0; a < 3; ++a) {
        g.n[a] = d.n[a];
        // a law end reads like a frozen one: ghosts clamp to its extra node
        g.bc_lo[a] = a < d.dim ? (d.bc_lo[a] == SFG_BC_LAW ? BC_FROZEN : d.bc_lo[a]) : BC_TRANSMISSIVE;
        g.bc_hi[a] = a < d.dim ? (d.bc_hi[a] == SFG_BC_LAW ? BC_FROZEN : d.bc_hi[a]) : BC_TRANSMISSIVE;
        if (a < d.dim) {  // transmissive and law boundary nodes and extra nodes are not advanced
            g.lo[a] = d.bc_lo[a] == SFG_BC_PERIODIC ? 0 : (d.bc_lo[a] == SFG_BC_LAW ? 2 : 1);
            g.hi[a] = d.bc_hi[a] == SFG_BC_PERIODIC ? d.n[a] : (d.bc_hi[a] == SFG_BC_LAW ? d.n[a] - 2 : d.n[a] - 1);
        } else {
            g.lo[a] = 0;
            g.hi[a] = 1;
        }
    }
    // Uniform Cartesian metrics exactly as the reference mesh yields them for
    // equal spacing (SF_mesh.cpp:283-339): J = dx dy dz, Jac = 1/J,
    // xi_x = (dy dz) Jac; face cofactor (SF_canonicalFace.h:94-103) =
    // 0.5 (xi_x/Jac + xi_x/Jac).
    const double hx = d.h[0], hy = d.h[1], hz = d.h[2];
    const double J = hx * hy * hz;
    g.jac = 1.0 / J;
    g.metric[0] = (hy * hz) * g.jac;
    g.metric[1] = (hx * hz) * g.jac;
    g.metric[2] = (hx * hy) * g.jac;
    for (int a = 0; a < 3; ++a) g.area[a] = 0.5 * (g.metric[a] / g.jac + g.metric[a] / g.jac);
    g.gamma = s->num.gamma;
    for (int a = 0; a < 3; ++a) g.h[a] = d.h[a];
    g.cfl = s->num.cfl;
    s->nodes = (long long)d.n[0] * d.n[1] * d.n[2];
    g.vs = (s->nodes + 31) / 32 * 32;
    build_law_view(s);
}

StageView stage_view(sfg_solver_s* s, int stage, bool residual_only, bool require_active) {
    StageView sv{};
    sv.clock = s->clock;
    sv.flags = s->flags;
    sv.counters = s->counting ? s->counters : nullptr;
    sv.time_id = s->num.time_recipe;
    sv.stage = stage;
    sv.q0 = s->qn;
    sv.r = s->r;
    sv.k = s->k;
    sv.require_active = require_active ? 1 : 0;
    if (residual_only) {
        sv.qs = s->qn;
        sv.qout = nullptr;
        return sv;
    }
    switch (s->num.time_recipe) {
    case T_EULER:
        sv.qs = s->qn;
        sv.qout = s->qa;
        break;
    case T_SSPRK3: {
        static const double base[3] = {0.0, 0.75, 1.0 / 3.0};
        static const double inc[3] = {1.0, 0.25, 2.0 / 3.0};
        sv.base = base[stage];
        sv.inc = inc[stage];
        const double* in[3] = {s->qn, s->qa, s->qb};
        double* out[3] = {s->qa, s->qb, s->qn};
        sv.qs = in[stage];
        sv.qout = out[stage];
        break;
    }
    default: {
        static const double inc[4] = {0.5, 0.5, 1.0, 0.0};
        sv.inc = inc[stage];
        const double* in[4] = {s->qn, s->qa, s->qb, s->qa};
        double* out[4] = {s->qa, s->qb, s->qa, s->qn};
        sv.qs = in[stage];
        sv.qout = out[stage];
        break;
    }
    }
    return sv;
}

// All axis sweeps of one stage (or of the residual alone).
// `cfl`: the launch that finishes the nodes also reduces the CFL minimum of
// the new state (the last stage of a step).
int enqueue_stage(sfg_solver_s* s, int stage, bool residual_only, bool require_active, bool cfl = false) {
    StageView sv = stage_view(s, stage, residual_only, require_active);
    const int dim = s->grid.dim;
    const int cfl_bit_all = cfl && !residual_only ? MODE_CFL : 0;
    if (s->has_laws) {
        // prepareBoundaryState before the RHS: the laws on the stage's input;
        // the previous application's values sit in the previous stage's input
        const double* old = stage == 0 || residual_only ? s->qn : stage_view(s, stage - 1, false, false).qs;
        CUDA_TRY(launch_law_fill(s->gv, s->lv, old, const_cast<double*>(sv.qs), s->clock, require_active ? 1 : 0,
                                 s->flags, s->stream));
    }
    if (s->gv.curv) {  // per-face geometry: face-flux launches per axis, then the stage
        sv.mode = MODE_FINAL | (residual_only ? MODE_RESIDUAL : 0) | cfl_bit_all;
        // 2-D: the fused tile unless variant 0 (face launches) is selected
        CUDA_TRY(launch_curv_stage(s->recipe->scheme, s->recipe->flux, s->num.precision == SFG_PREC_FP64,
                                   s->variant > 0, s->gv, sv, s->face_flux, s->stream));
        return SFG_OK;
    }
    const int cfl_bit = cfl && !residual_only ? MODE_CFL : 0;
    if (dim == 2 && s->variant > 0) {
        sv.mode = MODE_FINAL | (residual_only ? MODE_RESIDUAL : 0) | cfl_bit;
        CUDA_TRY(launch_tile2d(s->variant, s->recipe->scheme, s->recipe->flux, s->num.precision == SFG_PREC_FP64,
                               s->gv, sv, s->stream));
        return SFG_OK;
    }
    if (dim == 3 && s->variant > 0) {
        sv.mode = MODE_FINAL | (residual_only ? MODE_RESIDUAL : 0) | cfl_bit;
        CUDA_TRY(launch_tile3d(s->recipe->scheme, s->recipe->flux, s->num.precision == SFG_PREC_FP64, s->gv, sv,
                               s->stream));
        return SFG_OK;
    }
    if (dim == 1 && s->variant > 0) {
        sv.mode = MODE_FINAL | (residual_only ? MODE_RESIDUAL : 0) | cfl_bit;
        CUDA_TRY(launch_tile1d(s->recipe->scheme, s->recipe->flux, s->num.precision == SFG_PREC_FP64, s->gv, sv,
                               s->stream));
        return SFG_OK;
    }
    for (int axis = 0; axis < dim; ++axis) {
        sv.mode = (axis > 0 ? MODE_READ_R : 0) | (axis == dim - 1 ? MODE_FINAL | cfl_bit : 0) |
                  (residual_only && axis == dim - 1 ? MODE_RESIDUAL : 0);
        CUDA_TRY(launch_sweep(s->recipe->scheme, s->recipe->flux, s->num.precision == SFG_PREC_FP64, axis, s->gv,
                              sv, s->stream));
    }
    return SFG_OK;
}

// FlowStepCommit's boundary application on the last stage's output (before
// the Euler copy-back, which then carries it into qn).
int enqueue_commit_laws(sfg_solver_s* s, bool require_active) {
    if (!s->has_laws) return SFG_OK;
    const StageView last = stage_view(s, stage_count(s->num.time_recipe) - 1, false, false);
    CUDA_TRY(launch_law_fill(s->gv, s->lv, last.qs, last.qout, s->clock, require_active ? 1 : 0, s->flags,
                             s->stream));
    return SFG_OK;
}

// Euler writes to qa; the committed state lives in qn.
int enqueue_post_step(sfg_solver_s* s) {
    if (s->num.time_recipe == T_EULER)
        CUDA_TRY(cudaMemcpyAsync(s->qn, s->qa, sizeof(double) * 5 * s->gv.vs, cudaMemcpyDeviceToDevice, s->stream));
    return SFG_OK;
}

// One full step with the CFL dt computed and clipped on device.  The CFL
// minimum of the step's result is reduced by its last stage (MODE_CFL) and
// marked ready by the commit, so the next step's dt_kernel returns at once;
// dt_kernel reads the state only when nothing reduced it (first step after
// an upload, a host-driven stage or the start of sfg_advance).
int enqueue_cfl_step(sfg_solver_s* s, bool require_active) {
    CUDA_TRY(launch_dt(s->gv, s->qn, s->clock, s->flags, 1, s->stream));
    CUDA_TRY(launch_finalize_dt(s->clock, s->flags, s->stream));
    // FlowStepPrepare opens the step (before its dt in the reference; the dt
    // reads solved nodes only, which the laws never write)
    if (s->has_laws)
        CUDA_TRY(launch_law_fill(s->gv, s->lv, s->qn, s->qn, s->clock, require_active ? 1 : 0, s->flags, s->stream));
    const int ns = stage_count(s->num.time_recipe);
    for (int st = 0; st < ns; ++st) {
        int rc = enqueue_stage(s, st, false, require_active, st == ns - 1);
        if (rc) return rc;
    }
    int rc = enqueue_commit_laws(s, require_active);
    if (rc) return rc;
    if (s->num.time_recipe == T_EULER) {
        // guarded copy: only when the step ran (graph-safe: copy unconditionally
        // is wrong once the run has stopped), so Euler keeps its own kernel path
        int rc = enqueue_post_step(s);
        if (rc) return rc;
    }
    CUDA_TRY(launch_commit(s->clock, s->dt_log, s->dt_log_cap, 1, s->stream));
    return SFG_OK;
}

int sync_and_check(sfg_solver_s* s) {
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    unsigned bits = 0;
    CUDA_TRY(cudaMemcpy(&bits, s->flags, sizeof bits, cudaMemcpyDeviceToHost));
    if (bits & FLAG_TENO_CUTOFF) return fail(SFG_ERR_TENO_CUTOFF, "TENO5 rejected all sub-stencils (flags 0x%x)", bits);
    if (bits) return fail(SFG_ERR_STATE, "invalid state on device (flags 0x%x)", bits);
    return SFG_OK;
}

int push_clock(sfg_solver_s* s) {
    CUDA_TRY(cudaMemcpyAsync(s->clock, s->host_clock, sizeof(Clock), cudaMemcpyHostToDevice, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    return SFG_OK;
}

int pull_clock(sfg_solver_s* s) {
    CUDA_TRY(cudaMemcpyAsync(s->host_clock, s->clock, sizeof(Clock), cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    return SFG_OK;
}

const double kInf = std::numeric_limits<double>::infinity();

void reset_clock(Clock* c, double t) {
    std::memset(c, 0, sizeof *c);
    c->t = t;
    c->t_end = kInf;
    c->next_out = kInf;
    c->write_interval = 0.0;
    c->max_dt = kInf;
    c->limit = kInf;
    c->dt_bits = 0x7FEFFFFFFFFFFFFFull;
    c->max_steps = std::numeric_limits<long long>::max();
}

// Host-layout helpers: reference Field storage (ng ghosts on every axis) <->
// node block.  Ghost values follow the same laws the kernels read through.
long long field_extent(const sfg_solver_s* s, int a) { return s->grid.n[a] + 2LL * s->ng; }

// Index map of the device grid (same laws as map_index in the kernels).
int map_host(int i, int n, int bl, int bh) {
    if (bl == SFG_BC_PERIODIC) {
        while (i < 0) i += n;
    } else if (bl == SFG_BC_FROZEN || bl == SFG_BC_LAW) {
        if (i < 0) i = 0;
    } else if (i < 1) {
        i = n > 1 ? 1 : 0;
    }
    if (bh == SFG_BC_PERIODIC) {
        while (i >= n) i -= n;
    } else if (bh == SFG_BC_FROZEN || bh == SFG_BC_LAW) {
        if (i > n - 1) i = n - 1;
    } else if (i > n - 2) {
        i = n > 1 ? n - 2 : 0;
    }
    return i;
}

// Caller node layout -> device node layout (AoS).  A frozen end's extra node
// takes the boundary node's value -- the reference initialises ghosts by
// clamping to the interior (SF_mesh.cpp:544) -- or 0 with `zero_extra`.
void nodes_to_device_layout(const sfg_solver_s* s, const double* pub, double* dev, bool zero_extra) {
    const int* N = s->ig.n;
    const int* P = s->grid.n;
    for (int k = 0; k < N[2]; ++k)
        for (int j = 0; j < N[1]; ++j)
            for (int i = 0; i < N[0]; ++i) {
                int c[3] = {i - s->off_lo[0], j - s->off_lo[1], k - s->off_lo[2]};
                bool extra = false;
                for (int a = 0; a < 3; ++a) {
                    if (c[a] < 0) c[a] = 0, extra = true;
                    if (c[a] >= P[a]) c[a] = P[a] - 1, extra = true;
                }
                double* out = dev + (((long long)k * N[1] + j) * N[0] + i) * 5;
                if (extra && zero_extra) {
                    std::memset(out, 0, 5 * sizeof(double));
                    continue;
                }
                std::memcpy(out, pub + (((long long)c[2] * P[1] + c[1]) * P[0] + c[0]) * 5, 5 * sizeof(double));
            }
}

// Device node layout -> caller node layout (drops the frozen extra nodes).
void nodes_from_device_layout(const sfg_solver_s* s, const double* dev, double* pub) {
    const int* N = s->ig.n;
    const int* P = s->grid.n;
    for (int k = 0; k < P[2]; ++k)
        for (int j = 0; j < P[1]; ++j)
            for (int i = 0; i < P[0]; ++i) {
                const long long src =
                    (((long long)(k + s->off_lo[2]) * N[1] + (j + s->off_lo[1])) * N[0] + (i + s->off_lo[0])) * 5;
                std::memcpy(pub + (((long long)k * P[1] + j) * P[0] + i) * 5, dev + src, 5 * sizeof(double));
            }
}

}  // namespace

namespace sfg {

// What is wrong with a law, or nullptr (the checks of sfg_set_boundary_law).
const char* law_problem(const sfg_boundary_law& law) {
    for (int k : {law.rho, law.velocity, law.pressure})
        if (k != SFG_LAW_ZERO_GRADIENT && k != SFG_LAW_FIXED_VALUE && k != SFG_LAW_SYMMETRY)
            return "unknown field law";
    auto finite = [](double v) { return std::isfinite(v); };
    if (!finite(law.rho_value) || !finite(law.pressure_value) || !finite(law.velocity_value[0]) ||
        !finite(law.velocity_value[1]) || !finite(law.velocity_value[2]))
        return "law values must be finite";
    if (law.rho == SFG_LAW_FIXED_VALUE && !(law.rho_value > 0.0)) return "fixedValue density must be > 0";
    if (law.pressure == SFG_LAW_FIXED_VALUE && !(law.pressure_value > 0.0)) return "fixedValue pressure must be > 0";
    return nullptr;
}

// The law view and the state-cache replay of a grid that is not a solver of
// its own (a batched grid): `G` in the caller's layout, `gv` its device view
// with the extra end nodes (offset off_lo), ng the Field's ghost layers.
void grid_law_view(const sfg_grid_desc& G, const GridView& gv, const int off_lo[3], const sfg_boundary_law* laws,
                   int ng, LawView& lv, std::vector<unsigned char>& codes) {
    make_law_view(G, gv, laws, lv);
    simulate_law_cache(lv, G, gv, off_lo, ng, codes);
}

}  // namespace sfg

extern "C" {

const char* sfg_last_error(void) { return g_error.c_str(); }

int sfg_version(int* major, int* minor) {
    if (major) *major = 0;
    if (minor) *minor = 1;
    return SFG_OK;
}

const char* sfg_recipe_name(int recipe) {
    const RecipeInfo* r = find_recipe(recipe);
    return r ? r->name : nullptr;
}

int sfg_recipe_from_name(const char* name, int* recipe) {
    if (!name || !recipe) return fail(SFG_ERR_ARG, "null argument");
    for (const auto& r : kRecipes)
        if (std::strcmp(r.name, name) == 0) {
            *recipe = r.id;
            return SFG_OK;
        }
    return fail(SFG_ERR_ARG, "convection recipe '%s' is not provided on the GPU", name);
}

int sfg_create(const sfg_grid_desc* grid, const sfg_numerics_desc* numerics, void* stream, sfg_solver* out) {
    if (!out) return fail(SFG_ERR_ARG, "null output handle");
    *out = nullptr;
    const RecipeInfo* recipe = nullptr;
    int rc = validate(grid, numerics, &recipe);
    if (rc) return rc;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(SFG_ERR_CUDA, "no CUDA device: the B200 provider has no CPU fallback");
    auto* s = new sfg_solver_s;
    s->grid = *grid;
    s->num = *numerics;
    if (!(s->num.max_dt > 0.0)) s->num.max_dt = kInf;
    s->recipe = recipe;
    s->ng = ghost_layers(recipe->scheme);
    make_view(s);
    s->variant = grid->dim == 1 ? 2 : grid->dim == 2 ? 1 : 0;
    cudaGetDevice(&s->device);
    auto cleanup = [&](int code) {
        sfg_destroy(s);
        return code;
    };
    if (stream) {
        s->stream = (cudaStream_t)stream;
    } else {
        if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess)
            return cleanup(fail(SFG_ERR_CUDA, "stream creation failed"));
        s->own_stream = true;
    }
    const size_t state_bytes = sizeof(double) * 5 * (size_t)s->gv.vs;
    double** bufs[] = {&s->qn, &s->qa, &s->qb, &s->r};
    for (double** b : bufs)
        if (cudaMalloc((void**)b, state_bytes) != cudaSuccess)
            return cleanup(fail(SFG_ERR_NOMEM, "device allocation of %zu bytes failed", state_bytes));
    if (s->num.time_recipe == T_RK4 && cudaMalloc((void**)&s->k, state_bytes) != cudaSuccess)
        return cleanup(fail(SFG_ERR_NOMEM, "device allocation failed"));
    if (cudaMalloc((void**)&s->staging, sizeof(double) * 5 * (size_t)s->nodes) != cudaSuccess ||
        cudaMalloc((void**)&s->clock, sizeof(Clock)) != cudaSuccess ||
        cudaMalloc((void**)&s->flags, 64) != cudaSuccess ||
        cudaMalloc((void**)&s->counters, 64) != cudaSuccess ||
        cudaMalloc((void**)&s->totals, 64) != cudaSuccess)
        return cleanup(fail(SFG_ERR_NOMEM, "device allocation failed"));
    if (cudaMallocHost((void**)&s->host_clock, sizeof(Clock)) != cudaSuccess)
        return cleanup(fail(SFG_ERR_NOMEM, "pinned allocation failed"));
    cudaMemsetAsync(s->flags, 0, 64, s->stream);
    cudaMemsetAsync(s->counters, 0, 64, s->stream);
    cudaMemsetAsync(s->qn, 0, state_bytes, s->stream);
    cudaMemsetAsync(s->qa, 0, state_bytes, s->stream);
    cudaMemsetAsync(s->qb, 0, state_bytes, s->stream);
    cudaMemsetAsync(s->r, 0, state_bytes, s->stream);
    reset_clock(s->host_clock, 0.0);
    s->host_clock->max_dt = s->num.max_dt;
    rc = push_clock(s);
    if (rc) return cleanup(rc);
    rc = upload_law_codes(s);
    if (rc) return cleanup(rc);
    *out = s;
    return SFG_OK;
}

int sfg_destroy(sfg_solver s) {
    if (!s) return SFG_OK;
    if (s->stream) cudaStreamSynchronize(s->stream);
    if (s->graph) cudaGraphExecDestroy(s->graph);
    for (double* p : {s->qn, s->qa, s->qb, s->r, s->k, s->staging, s->totals, s->dt_log})
        if (p) cudaFree(p);
    if (s->clock) cudaFree(s->clock);
    if (s->law_codes) cudaFree(s->law_codes);
    for (double* p : {s->node_metrics, s->face_geom, s->face_flux})
        if (p) cudaFree(p);
    if (s->flags) cudaFree(s->flags);
    if (s->counters) cudaFree(s->counters);
    if (s->host_clock) cudaFreeHost(s->host_clock);
    if (s->own_stream && s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return SFG_OK;
}

int sfg_set_boundary_law(sfg_solver s, int axis, int end, const sfg_boundary_law* law) {
    if (!s || !law) return fail(SFG_ERR_ARG, "null argument");
    if (axis < 0 || axis >= s->grid.dim || end < 0 || end > 1) return fail(SFG_ERR_ARG, "bad axis %d / end %d", axis, end);
    if ((end ? s->grid.bc_hi[axis] : s->grid.bc_lo[axis]) != SFG_BC_LAW)
        return fail(SFG_ERR_ARG, "axis %d end %d is not a SFG_BC_LAW end", axis, end);
    if (const char* why = sfg::law_problem(*law)) return fail(SFG_ERR_ARG, "%s", why);
    s->laws[2 * axis + end] = *law;
    build_law_view(s);
    if (s->graph) {  // the captured launches hold the previous laws
        cudaGraphExecDestroy(s->graph);
        s->graph = nullptr;
    }
    return upload_law_codes(s);
}

// Caller metrics (10 per node: Jac, xi_x, xi_y, xi_z, eta_x, eta_y, eta_z,
// zeta_x, zeta_y, zeta_z) in the node or Field layout -> device SoA over the
// device grid (extra nodes: the Field's first ghost layer, or the boundary
// node's metrics in the node layout).
static void metrics_to_device(const sfg_solver_s* s, const double* host, int layout, std::vector<double>& soa) {
    const int* N = s->ig.n;
    const int* P = s->grid.n;
    const long long vs = s->gv.vs;
    soa.assign((size_t)10 * vs, 0.0);
    const long long mx = field_extent(s, 0), my = field_extent(s, 1);
    for (int k = 0; k < N[2]; ++k)
        for (int j = 0; j < N[1]; ++j)
            for (int i = 0; i < N[0]; ++i) {
                int c[3] = {i - s->off_lo[0], j - s->off_lo[1], k - s->off_lo[2]};
                const double* src;
                if (layout == SFG_LAYOUT_FIELD) {
                    const long long fi = c[0] + s->ng, fj = c[1] + s->ng, fk = c[2] + s->ng;
                    src = host + ((fk * my + fj) * mx + fi) * 10;
                } else {
                    for (int a = 0; a < 3; ++a) c[a] = c[a] < 0 ? 0 : (c[a] >= P[a] ? P[a] - 1 : c[a]);
                    src = host + (((long long)c[2] * P[1] + c[1]) * P[0] + c[0]) * 10;
                }
                const long long node = ((long long)k * N[1] + j) * N[0] + i;
                for (int m = 0; m < 10; ++m) soa[(size_t)(m * vs + node)] = src[m];
            }
}

int sfg_set_metrics(sfg_solver s, const double* host, int layout) {
    if (!s || !host) return fail(SFG_ERR_ARG, "null argument");
    if (layout != SFG_LAYOUT_NODES && layout != SFG_LAYOUT_FIELD) return fail(SFG_ERR_ARG, "unknown layout %d", layout);
    if (s->recipe->flux == LAXW)
        return fail(SFG_ERR_ARG, "%s: Lax-Wendroff needs node coordinates; curvilinear grids take the other fluxes",
                    s->recipe->name);
    std::vector<double> soa;
    metrics_to_device(s, host, layout, soa);
    for (double x : soa)
        if (!std::isfinite(x)) return fail(SFG_ERR_ARG, "metrics must be finite");
    const size_t vsb = sizeof(double) * (size_t)s->gv.vs;
    if (!s->node_metrics && (cudaMalloc((void**)&s->node_metrics, 10 * vsb) != cudaSuccess ||
                             cudaMalloc((void**)&s->face_geom, 12 * vsb) != cudaSuccess ||
                             cudaMalloc((void**)&s->face_flux, 15 * vsb) != cudaSuccess))
        return fail(SFG_ERR_NOMEM, "device allocation of the metric arrays failed");
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    // every transfer on the solver's stream: it is non-blocking, so a copy or
    // memset on the legacy stream would not be ordered before the geometry
    // kernel (a late memset of face_geom would wipe the face areas)
    CUDA_TRY(cudaMemcpyAsync(s->node_metrics, soa.data(), 10 * vsb, cudaMemcpyHostToDevice, s->stream));
    CUDA_TRY(cudaMemsetAsync(s->face_geom, 0, 12 * vsb, s->stream));
    CUDA_TRY(cudaMemsetAsync(s->face_flux, 0, 15 * vsb, s->stream));
    GridView g = s->gv;
    double* geom[3] = {s->face_geom, s->face_geom + 4 * s->gv.vs, s->face_geom + 8 * s->gv.vs};
    CUDA_TRY(cudaMemsetAsync(s->flags, 0, 64, s->stream));
    CUDA_TRY(launch_curv_geometry(g, s->node_metrics, geom, s->flags, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    unsigned bits = 0;
    CUDA_TRY(cudaMemcpy(&bits, s->flags, sizeof bits, cudaMemcpyDeviceToHost));
    if (bits) return fail(SFG_ERR_ARG, "metrics give a degenerate face (zero Jac or zero area)");
    s->gv.curv = 1;
    s->gv.node_jac = s->node_metrics;
    s->gv.node_metric = s->node_metrics + s->gv.vs;
    for (int a = 0; a < 3; ++a) s->gv.geom[a] = geom[a];
    if (s->graph) {  // the captured launches hold the previous grid view
        cudaGraphExecDestroy(s->graph);
        s->graph = nullptr;
    }
    return SFG_OK;
}

int sfg_apply_boundary(sfg_solver s) {
    if (!s) return fail(SFG_ERR_ARG, "null solver");
    if (!s->has_laws) return SFG_OK;
    CUDA_TRY(launch_law_fill(s->gv, s->lv, s->qn, s->qn, s->clock, 0, s->flags, s->stream));
    return sync_and_check(s);
}

int sfg_ghost_layers(sfg_solver s, int* ng) {
    if (!s || !ng) return fail(SFG_ERR_ARG, "null argument");
    *ng = s->ng;
    return SFG_OK;
}

int sfg_state_size(sfg_solver s, int layout, size_t* count) {
    if (!s || !count) return fail(SFG_ERR_ARG, "null argument");
    if (layout == SFG_LAYOUT_NODES) *count = 5 * (size_t)s->pub_nodes;
    else if (layout == SFG_LAYOUT_FIELD)
        *count = 5 * (size_t)(field_extent(s, 0) * field_extent(s, 1) * field_extent(s, 2));
    else return fail(SFG_ERR_ARG, "unknown layout %d", layout);
    return SFG_OK;
}

static int upload_nodes_host(sfg_solver s, const double* nodes_aos) {
    CUDA_TRY(cudaMemcpyAsync(s->staging, nodes_aos, sizeof(double) * 5 * s->nodes, cudaMemcpyHostToDevice, s->stream));
    CUDA_TRY(launch_aos_to_soa(s->staging, s->qn, s->nodes, s->gv.vs, s->stream));
    if (s->frozen) {
        // Stage kernels write solved nodes only, and stage outputs (and the
        // Euler copy-back qa -> qn) are read as the next state: every stage
        // buffer must hold the frozen ghost value in its extra nodes.
        const size_t bytes = sizeof(double) * 5 * (size_t)s->gv.vs;
        CUDA_TRY(cudaMemcpyAsync(s->qa, s->qn, bytes, cudaMemcpyDeviceToDevice, s->stream));
        CUDA_TRY(cudaMemcpyAsync(s->qb, s->qn, bytes, cudaMemcpyDeviceToDevice, s->stream));
    }
    return SFG_OK;
}

static int reset_time(sfg_solver s, double time) {
    reset_clock(s->host_clock, time);
    s->host_clock->max_dt = s->num.max_dt;
    s->next_stage = 0;
    CUDA_TRY(cudaMemsetAsync(s->flags, 0, 64, s->stream));
    return push_clock(s);
}

int sfg_upload(sfg_solver s, const double* host, int layout, double time) {
    sfg::NvtxRange nvtx_("sfg_upload");
    if (!s || !host) return fail(SFG_ERR_ARG, "null argument");
    if (layout == SFG_LAYOUT_NODES && !s->frozen) {
        int rc = upload_nodes_host(s, host);
        if (rc) return rc;
    } else if (layout == SFG_LAYOUT_NODES) {
        std::vector<double> tmp(5 * (size_t)s->nodes);
        nodes_to_device_layout(s, host, tmp.data(), false);
        int rc = upload_nodes_host(s, tmp.data());
        if (rc) return rc;
        CUDA_TRY(cudaStreamSynchronize(s->stream));
    } else if (layout == SFG_LAYOUT_FIELD) {
        // device node (i, j, k) <- Field entry at caller node (i - off) + ng:
        // a frozen end's extra node reads the Field's first ghost layer
        std::vector<double> tmp(5 * (size_t)s->nodes);
        const long long mx = field_extent(s, 0), my = field_extent(s, 1);
        const int ng = s->ng;
        const int* N = s->ig.n;
        for (int k = 0; k < N[2]; ++k)
            for (int j = 0; j < N[1]; ++j)
                for (int i = 0; i < N[0]; ++i) {
                    const long long fi = i - s->off_lo[0] + ng, fj = j - s->off_lo[1] + ng, fk = k - s->off_lo[2] + ng;
                    const long long src = ((fk * my + fj) * mx + fi) * 5;
                    const long long dst = (((long long)k * N[1] + j) * N[0] + i) * 5;
                    std::memcpy(&tmp[dst], host + src, 5 * sizeof(double));
                }
        int rc = upload_nodes_host(s, tmp.data());
        if (rc) return rc;
        CUDA_TRY(cudaStreamSynchronize(s->stream));
    } else {
        return fail(SFG_ERR_ARG, "unknown layout %d", layout);
    }
    return reset_time(s, time);
}

int sfg_restore(sfg_solver s, const double* host, int layout, double time, int64_t steps) {
    sfg::NvtxRange nvtx_("sfg_restore");
    if (!s || !host) return fail(SFG_ERR_ARG, "null argument");
    if (!std::isfinite(time)) return fail(SFG_ERR_ARG, "time must be finite");
    if (steps < 0) return fail(SFG_ERR_ARG, "steps must be >= 0");
    if (int rc = sfg_upload(s, host, layout, time)) return rc;
    s->host_clock->steps = steps;
    return push_clock(s);
}

int sfg_upload_device(sfg_solver s, const double* dev_nodes_aos, double time) {
    if (!s || !dev_nodes_aos) return fail(SFG_ERR_ARG, "null argument");
    if (s->frozen) return fail(SFG_ERR_ARG, "frozen boundary ends need sfg_upload (host layouts)");
    CUDA_TRY(launch_aos_to_soa(dev_nodes_aos, s->qn, s->nodes, s->gv.vs, s->stream));
    return reset_time(s, time);
}

int sfg_download_device(sfg_solver s, double* dev_nodes_aos) {
    if (!s || !dev_nodes_aos) return fail(SFG_ERR_ARG, "null argument");
    if (s->frozen) return fail(SFG_ERR_ARG, "frozen boundary ends need sfg_download (host layouts)");
    CUDA_TRY(launch_soa_to_aos(s->gv, s->qn, dev_nodes_aos, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    return SFG_OK;
}

int sfg_download(sfg_solver s, double* host, int layout) {
    sfg::NvtxRange nvtx_("sfg_download");
    if (!s || !host) return fail(SFG_ERR_ARG, "null argument");
    CUDA_TRY(launch_soa_to_aos(s->gv, s->qn, s->staging, s->stream));
    if (layout == SFG_LAYOUT_NODES && !s->frozen) {
        CUDA_TRY(cudaMemcpyAsync(host, s->staging, sizeof(double) * 5 * s->nodes, cudaMemcpyDeviceToHost, s->stream));
        CUDA_TRY(cudaStreamSynchronize(s->stream));
        return SFG_OK;
    }
    if (layout != SFG_LAYOUT_NODES && layout != SFG_LAYOUT_FIELD) return fail(SFG_ERR_ARG, "unknown layout %d", layout);
    std::vector<double> tmp(5 * (size_t)s->nodes);
    CUDA_TRY(cudaMemcpyAsync(tmp.data(), s->staging, sizeof(double) * 5 * s->nodes, cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    if (layout == SFG_LAYOUT_NODES) {
        nodes_from_device_layout(s, tmp.data(), host);
        return SFG_OK;
    }
    // Field entry (i, j, k) <- device node map(caller node (i - ng) + off):
    // ghosts follow the boundary laws, a frozen end's ghosts its extra node
    const long long mx = field_extent(s, 0), my = field_extent(s, 1), mz = field_extent(s, 2);
    const int ng = s->ng;
    const int* N = s->ig.n;
    for (long long k = 0; k < mz; ++k)
        for (long long j = 0; j < my; ++j)
            for (long long i = 0; i < mx; ++i) {
                int c[3] = {(int)i - ng, (int)j - ng, (int)k - ng};
                for (int a = 0; a < 3; ++a) {
                    if (a < s->ig.dim) {
                        c[a] = map_host(c[a] + s->off_lo[a], N[a], s->ig.bc_lo[a], s->ig.bc_hi[a]);
                    } else {
                        c[a] = c[a] < 0 ? 0 : (c[a] >= N[a] ? N[a] - 1 : c[a]);
                    }
                }
                const long long src = (((long long)c[2] * N[1] + c[1]) * N[0] + c[0]) * 5;
                std::memcpy(host + ((k * my + j) * mx + i) * 5, &tmp[src], 5 * sizeof(double));
            }
    return SFG_OK;
}

int sfg_compute_dt(sfg_solver s, double limit, double* dt) {
    sfg::NvtxRange nvtx_("sfg_compute_dt");
    if (!s || !dt) return fail(SFG_ERR_ARG, "null argument");
    CUDA_TRY(launch_reset_min(s->clock, s->stream));
    CUDA_TRY(launch_dt(s->gv, s->qn, s->clock, s->flags, 0, s->stream));
    int rc = pull_clock(s);
    if (rc) return rc;
    double v;
    unsigned long long bits = s->host_clock->dt_bits;
    std::memcpy(&v, &bits, sizeof v);
    if (s->num.max_dt < v) v = s->num.max_dt;
    if (limit > 0.0 && limit < v) v = limit;
    *dt = v;
    return SFG_OK;
}

int sfg_stage(sfg_solver s, int stage, double dt) {
    sfg::NvtxRange nvtx_("sfg_stage");
    if (!s) return fail(SFG_ERR_ARG, "null solver");
    const int ns = stage_count(s->num.time_recipe);
    if (stage != s->next_stage || stage < 0 || stage >= ns)
        return fail(SFG_ERR_ARG, "explicit stage %d out of order (expected %d)", stage, s->next_stage);
    if (!(dt > 0.0) || !std::isfinite(dt)) return fail(SFG_ERR_ARG, "dt must be finite and > 0");
    if (stage == 0) s->stage_dt = dt;
    else if (dt != s->stage_dt) return fail(SFG_ERR_ARG, "dt changed inside a step");
    CUDA_TRY(launch_set_dt(s->clock, dt, s->stream));
    int rc = enqueue_stage(s, stage, false, false);
    if (rc) return rc;
    if (stage == ns - 1) {
        rc = enqueue_commit_laws(s, false);
        if (rc) return rc;
        rc = enqueue_post_step(s);
        if (rc) return rc;
        CUDA_TRY(launch_commit(s->clock, nullptr, 0, 0, s->stream));
        s->next_stage = 0;
    } else {
        s->next_stage = stage + 1;
    }
    return sync_and_check(s);
}

int sfg_step(sfg_solver s, double dt, double limit) {
    sfg::NvtxRange nvtx_("sfg_step");
    if (!s) return fail(SFG_ERR_ARG, "null solver");
    if (s->next_stage != 0) return fail(SFG_ERR_ARG, "a step is in progress (stage %d)", s->next_stage);
    if (dt > 0.0) {
        if (s->has_laws)  // FlowStepPrepare
            CUDA_TRY(launch_law_fill(s->gv, s->lv, s->qn, s->qn, s->clock, 0, s->flags, s->stream));
        for (int st = 0; st < stage_count(s->num.time_recipe); ++st) {
            s->next_stage = st;
            int rc = sfg_stage(s, st, dt);
            if (rc) {
                s->next_stage = 0;
                return rc;
            }
        }
        return SFG_OK;
    }
    // CFL step on device; one-shot limit through the clock
    s->host_clock->t_end = kInf;
    s->host_clock->max_steps = std::numeric_limits<long long>::max();
    int rc = pull_clock(s);
    if (rc) return rc;
    s->host_clock->t_end = kInf;
    s->host_clock->max_steps = std::numeric_limits<long long>::max();
    s->host_clock->limit = limit > 0.0 ? limit : kInf;
    s->host_clock->dt_bits = 0x7FEFFFFFFFFFFFFFull;
    s->host_clock->dt_ready = 0;
    s->host_clock->write_interval = 0.0;
    s->host_clock->next_out = kInf;
    rc = push_clock(s);
    if (rc) return rc;
    rc = enqueue_cfl_step(s, false);
    if (rc) return rc;
    return sync_and_check(s);
}

// sfg_advance on the CUDA-graph path: graphs of `graph_steps` CFL steps,
// relaunched until the clock stops.  `ms`: device time of the launches.
static int advance_graph(sfg_solver_s* s, int graph_steps, float* ms) {
    Clock* hc = s->host_clock;
    if (!s->graph || s->graph_steps != graph_steps) {
        if (s->graph) cudaGraphExecDestroy(s->graph);
        s->graph = nullptr;
        cudaGraph_t g;
        CUDA_TRY(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
        int crc = SFG_OK;
        for (int i = 0; i < graph_steps && !crc; ++i) crc = enqueue_cfl_step(s, true);
        cudaError_t e = cudaStreamEndCapture(s->stream, &g);
        if (crc) return crc;
        if (e != cudaSuccess) return fail(SFG_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
        e = cudaGraphInstantiate(&s->graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return fail(SFG_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
        s->graph_steps = graph_steps;
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s->stream);
    for (;;) {
        CUDA_TRY(cudaGraphLaunch(s->graph, s->stream));
        CUDA_TRY(cudaMemcpyAsync(hc, s->clock, sizeof(Clock), cudaMemcpyDeviceToHost, s->stream));
        CUDA_TRY(cudaStreamSynchronize(s->stream));
        unsigned bits = 0;
        CUDA_TRY(cudaMemcpy(&bits, s->flags, sizeof bits, cudaMemcpyDeviceToHost));
        if (bits) break;
        if (!hc->active || hc->steps >= hc->max_steps) break;
    }
    cudaEventRecord(e1, s->stream);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return SFG_OK;
}

// sfg_advance of a small 1-D FP64 grid in the whole-run cluster kernel
// (sfg_cluster1d.cu), relaunched every `launch_steps` steps until the clock
// stops.  `ran` stays false when the device cannot place the cluster; the
// caller then takes the graph path from the same state.
static int advance_cluster(sfg_solver_s* s, float* ms, bool* ran) {
    Clock* hc = s->host_clock;
    ClusterRun run{};
    run.stages = stage_count(s->num.time_recipe);
    for (int st = 0; st < run.stages; ++st) run.sv[st] = stage_view(s, st, false, false);
    run.clock = s->clock;
    run.dt_log = s->dt_log;
    run.dt_cap = s->dt_log_cap;
    run.flags = s->flags;
    run.launch_steps = 4096;
    cudaEvent_t e0, e1;
    CUDA_TRY(cudaEventCreate(&e0));
    CUDA_TRY(cudaEventCreate(&e1));
    CUDA_TRY(cudaEventRecord(e0, s->stream));
    for (bool first = true;; first = false) {
        cudaError_t e = launch_cluster1d(s->recipe->scheme, s->recipe->flux, s->gv, run, s->stream);
        if (e != cudaSuccess) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            if (first) {  // not placed: nothing ran
                (void)cudaGetLastError();
                return SFG_OK;
            }
            return fail(SFG_ERR_CUDA, "cluster run: %s", cudaGetErrorString(e));
        }
        CUDA_TRY(cudaMemcpyAsync(hc, s->clock, sizeof(Clock), cudaMemcpyDeviceToHost, s->stream));
        CUDA_TRY(cudaStreamSynchronize(s->stream));
        unsigned bits = 0;
        CUDA_TRY(cudaMemcpy(&bits, s->flags, sizeof bits, cudaMemcpyDeviceToHost));
        if (bits || !hc->active || hc->steps >= hc->max_steps) break;
    }
    CUDA_TRY(cudaEventRecord(e1, s->stream));
    CUDA_TRY(cudaEventSynchronize(e1));
    cudaEventElapsedTime(ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *ran = true;
    return SFG_OK;
}

int sfg_advance(sfg_solver s, double t_end, int64_t max_steps, double write_interval, int graph_steps,
                double* dt_out, int64_t dt_capacity, sfg_stats* stats) {
    sfg::NvtxRange nvtx_("sfg_advance");
    if (!s) return fail(SFG_ERR_ARG, "null solver");
    if (s->next_stage != 0) return fail(SFG_ERR_ARG, "a step is in progress");
    if (!(t_end == t_end)) return fail(SFG_ERR_ARG, "t_end is NaN");
    if (graph_steps <= 0) graph_steps = 32;
    int rc = pull_clock(s);
    if (rc) return rc;
    Clock* hc = s->host_clock;
    const long long steps0 = hc->steps;
    hc->t_end = t_end;
    hc->max_steps = max_steps > 0 ? steps0 + max_steps : std::numeric_limits<long long>::max();
    hc->write_interval = write_interval > 0.0 ? write_interval : 0.0;
    hc->next_out = write_interval > 0.0 ? hc->t + write_interval : kInf;
    hc->limit = kInf;
    hc->log_base = steps0;
    hc->dt_bits = 0x7FEFFFFFFFFFFFFFull;
    hc->dt_ready = 0;  // the first step reduces the CFL minimum itself
    // dt log buffer
    const long long want = dt_out && dt_capacity > 0 ? dt_capacity : 0;
    if (want > s->dt_log_cap) {
        if (s->dt_log) cudaFree(s->dt_log);
        s->dt_log = nullptr;
        s->dt_log_cap = 0;
        if (s->graph) {
            cudaGraphExecDestroy(s->graph);
            s->graph = nullptr;
        }
        if (cudaMalloc((void**)&s->dt_log, sizeof(double) * want) != cudaSuccess)
            return fail(SFG_ERR_NOMEM, "dt log allocation failed");
        s->dt_log_cap = want;
    }
    rc = push_clock(s);
    if (rc) return rc;
    float ms = 0.f;
    bool ran = false;
    if (s->grid.dim == 1 && s->variant == 2 && !s->has_laws &&
        cluster1d_eligible(s->gv, s->recipe->flux, s->num.precision == SFG_PREC_FP64)) {
        rc = advance_cluster(s, &ms, &ran);
        if (rc) return rc;
    }
    if (!ran) {
        rc = advance_graph(s, graph_steps, &ms);
        if (rc) return rc;
    }
    const long long done = hc->steps - steps0;
    if (dt_out && want > 0) {
        const long long n = done < want ? done : want;
        if (n > 0) CUDA_TRY(cudaMemcpy(dt_out, s->dt_log, sizeof(double) * n, cudaMemcpyDeviceToHost));
    }
    if (stats) {
        stats->steps = done;
        stats->time = hc->t;
        stats->last_dt = hc->dt;
        stats->device_ms = ms;
        unsigned bits = 0;
        cudaMemcpy(&bits, s->flags, sizeof bits, cudaMemcpyDeviceToHost);
        stats->status_bits = bits;
        unsigned long long cnt[2] = {0, 0};
        cudaMemcpy(cnt, s->counters, sizeof cnt, cudaMemcpyDeviceToHost);
        stats->teno_cores = cnt[0];
        stats->teno_cut = cnt[1];
    }
    // restore one-shot fields for later single steps
    hc->t_end = kInf;
    hc->max_steps = std::numeric_limits<long long>::max();
    hc->write_interval = 0.0;
    hc->next_out = kInf;
    hc->active = 0;
    rc = push_clock(s);
    if (rc) return rc;
    return sync_and_check(s);
}

int sfg_residual(sfg_solver s, double* host_nodes_aos) {
    sfg::NvtxRange nvtx_("sfg_residual");
    if (!s || !host_nodes_aos) return fail(SFG_ERR_ARG, "null argument");
    CUDA_TRY(cudaMemsetAsync(s->r, 0, sizeof(double) * 5 * s->gv.vs, s->stream));
    int rc = enqueue_stage(s, 0, true, false);
    if (rc) return rc;
    // unsolved nodes are reported as 0: copy R without boundary mapping
    GridView raw = s->gv;
    for (int a = 0; a < 3; ++a) raw.bc_lo[a] = raw.bc_hi[a] = BC_PERIODIC;  // identity mapping inside [0,n)
    raw.dim = 0;
    CUDA_TRY(launch_soa_to_aos(raw, s->r, s->staging, s->stream));
    if (!s->frozen) {
        CUDA_TRY(cudaMemcpyAsync(host_nodes_aos, s->staging, sizeof(double) * 5 * s->nodes, cudaMemcpyDeviceToHost,
                                 s->stream));
        return sync_and_check(s);
    }
    std::vector<double> tmp(5 * (size_t)s->nodes);
    CUDA_TRY(cudaMemcpyAsync(tmp.data(), s->staging, sizeof(double) * 5 * s->nodes, cudaMemcpyDeviceToHost, s->stream));
    rc = sync_and_check(s);
    if (rc) return rc;
    nodes_from_device_layout(s, tmp.data(), host_nodes_aos);
    return SFG_OK;
}

int sfg_stage_with_residual(sfg_solver s, int stage, double dt, const double* host_residual) {
    if (!s || !host_residual) return fail(SFG_ERR_ARG, "null argument");
    const int ns = stage_count(s->num.time_recipe);
    if (stage != s->next_stage || stage < 0 || stage >= ns)
        return fail(SFG_ERR_ARG, "explicit stage %d out of order (expected %d)", stage, s->next_stage);
    std::vector<double> tmp;
    if (s->frozen) {  // the extra nodes carry no residual
        tmp.resize(5 * (size_t)s->nodes);
        nodes_to_device_layout(s, host_residual, tmp.data(), true);
        host_residual = tmp.data();
    }
    CUDA_TRY(cudaMemcpyAsync(s->staging, host_residual, sizeof(double) * 5 * s->nodes, cudaMemcpyHostToDevice,
                             s->stream));
    if (s->frozen) CUDA_TRY(cudaStreamSynchronize(s->stream));
    CUDA_TRY(launch_aos_to_soa(s->staging, s->r, s->nodes, s->gv.vs, s->stream));
    CUDA_TRY(launch_set_dt(s->clock, dt, s->stream));
    StageView sv = stage_view(s, stage, false, false);
    CUDA_TRY(launch_stage_from_residual(s->gv, sv, s->stream));
    if (stage == ns - 1) {
        int rc = enqueue_post_step(s);
        if (rc) return rc;
        CUDA_TRY(launch_commit(s->clock, nullptr, 0, 0, s->stream));
        s->next_stage = 0;
    } else {
        s->next_stage = stage + 1;
    }
    return sync_and_check(s);
}

int sfg_conserved_totals(sfg_solver s, double totals[5]) {
    if (!s || !totals) return fail(SFG_ERR_ARG, "null argument");
    CUDA_TRY(cudaMemsetAsync(s->totals, 0, 5 * sizeof(double), s->stream));
    // node volume: the cell volume, or J = 1 / Jac per node on curvilinear grids
    const double vol = s->gv.curv ? 1.0 : s->grid.h[0] * s->grid.h[1] * s->grid.h[2];
    CUDA_TRY(launch_totals(s->gv, s->qn, s->totals, vol, s->stream));
    CUDA_TRY(cudaMemcpyAsync(totals, s->totals, 5 * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    return SFG_OK;
}

int sfg_time(sfg_solver s, double* time, int64_t* steps) {
    if (!s) return fail(SFG_ERR_ARG, "null solver");
    int rc = pull_clock(s);
    if (rc) return rc;
    if (time) *time = s->host_clock->t;
    if (steps) *steps = s->host_clock->steps;
    return SFG_OK;
}

int sfg_status_word(sfg_solver s, uint32_t* bits, int clear) {
    if (!s || !bits) return fail(SFG_ERR_ARG, "null argument");
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    unsigned b = 0;
    CUDA_TRY(cudaMemcpy(&b, s->flags, sizeof b, cudaMemcpyDeviceToHost));
    *bits = b;
    if (clear) {
        CUDA_TRY(cudaMemsetAsync(s->flags, 0, sizeof b, s->stream));
        CUDA_TRY(cudaStreamSynchronize(s->stream));
    }
    return SFG_OK;
}

int sfg_set_counting(sfg_solver s, int enable) {
    if (!s) return fail(SFG_ERR_ARG, "null solver");
    if ((enable != 0) != s->counting && s->graph) {
        cudaGraphExecDestroy(s->graph);
        s->graph = nullptr;
    }
    s->counting = enable != 0;
    CUDA_TRY(cudaMemsetAsync(s->counters, 0, 16, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    return SFG_OK;
}

int sfg_time_sweeps(sfg_solver s, int stage, double dt, int repeats, float* ms_per_axis) {
    if (!s || !ms_per_axis) return fail(SFG_ERR_ARG, "null argument");
    if (stage < 0 || stage >= stage_count(s->num.time_recipe)) return fail(SFG_ERR_ARG, "bad stage %d", stage);
    if (repeats < 1) repeats = 1;
    const int dim = s->grid.dim;
    cudaEvent_t ev[4];
    for (auto& e : ev) CUDA_TRY(cudaEventCreate(&e));
    double acc[3] = {0, 0, 0};
    CUDA_TRY(launch_set_dt(s->clock, dt, s->stream));
    StageView sv = stage_view(s, stage, false, false);
    if (s->variant > 0 || s->gv.curv) {  // one stage operator (tiles, or the curvilinear launches)
        // `repeats` back-to-back launches captured as one CUDA graph, as the
        // stages run inside a step's graph: the events bracket the graph,
        // so host launch latency does not enter the per-launch time
        cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
        CUDA_TRY(cudaStreamIsCapturing(s->stream, &cap));
        cudaGraphExec_t exec = nullptr;
        if (s->stream != nullptr && cap == cudaStreamCaptureStatusNone) {
            cudaGraph_t graph;
            CUDA_TRY(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
            int rc = SFG_OK;
            for (int r = 0; r < repeats && !rc; ++r) rc = enqueue_stage(s, stage, false, false);
            const cudaError_t ce = cudaStreamEndCapture(s->stream, &graph);
            if (rc) return rc;
            CUDA_TRY(ce);
            const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
            cudaGraphDestroy(graph);
            CUDA_TRY(ie);
            CUDA_TRY(cudaGraphLaunch(exec, s->stream));  // warm
            CUDA_TRY(cudaEventRecord(ev[0], s->stream));
            CUDA_TRY(cudaGraphLaunch(exec, s->stream));
            CUDA_TRY(cudaEventRecord(ev[1], s->stream));
            CUDA_TRY(cudaEventSynchronize(ev[1]));
            cudaGraphExecDestroy(exec);
            float ms = 0.f;
            CUDA_TRY(cudaEventElapsedTime(&ms, ev[0], ev[1]));
            acc[0] = ms;
        } else {  // the legacy default stream cannot be captured: launch by launch
            for (int r = 0; r < repeats; ++r) {
                CUDA_TRY(cudaEventRecord(ev[0], s->stream));
                int rc = enqueue_stage(s, stage, false, false);
                if (rc) return rc;
                CUDA_TRY(cudaEventRecord(ev[1], s->stream));
                CUDA_TRY(cudaEventSynchronize(ev[1]));
                float ms = 0.f;
                CUDA_TRY(cudaEventElapsedTime(&ms, ev[0], ev[1]));
                acc[0] += ms;
            }
        }
        for (auto& e : ev) cudaEventDestroy(e);
        ms_per_axis[0] = (float)(acc[0] / repeats);
        ms_per_axis[1] = 0.f;
        CUDA_TRY(cudaMemsetAsync(s->flags, 0, 64, s->stream));
        CUDA_TRY(cudaStreamSynchronize(s->stream));
        return SFG_OK;
    }
    for (int r = 0; r < repeats; ++r) {
        CUDA_TRY(cudaEventRecord(ev[0], s->stream));
        for (int axis = 0; axis < dim; ++axis) {
            sv.mode = (axis > 0 ? MODE_READ_R : 0) | (axis == dim - 1 ? MODE_FINAL : 0);
            CUDA_TRY(launch_sweep(s->recipe->scheme, s->recipe->flux, s->num.precision == SFG_PREC_FP64, axis, s->gv,
                                  sv, s->stream));
            CUDA_TRY(cudaEventRecord(ev[axis + 1], s->stream));
        }
        CUDA_TRY(cudaEventSynchronize(ev[dim]));
        for (int axis = 0; axis < dim; ++axis) {
            float ms = 0.f;
            CUDA_TRY(cudaEventElapsedTime(&ms, ev[axis], ev[axis + 1]));
            acc[axis] += ms;
        }
    }
    for (auto& e : ev) cudaEventDestroy(e);
    for (int axis = 0; axis < dim; ++axis) ms_per_axis[axis] = (float)(acc[axis] / repeats);
    // the timed stage was not committed: state and flags are left as they were
    CUDA_TRY(cudaMemsetAsync(s->flags, 0, 64, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    return SFG_OK;
}

int sfg_teno_flip_rate(sfg_solver s, uint64_t* decisions, uint64_t* flips) {
    if (!s || !decisions || !flips) return fail(SFG_ERR_ARG, "null argument");
    *decisions = *flips = 0;
    if (s->recipe->scheme != TENO5) return SFG_OK;
    unsigned long long* out = reinterpret_cast<unsigned long long*>(s->totals);
    CUDA_TRY(cudaMemsetAsync(out, 0, 2 * sizeof(unsigned long long), s->stream));
    CUDA_TRY(launch_teno_flips(s->gv, s->qn, out, s->stream));
    unsigned long long h[2];
    CUDA_TRY(cudaMemcpyAsync(h, out, sizeof h, cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    *decisions = h[0];
    *flips = h[1];
    return SFG_OK;
}

int sfg_set_kernel_variant(sfg_solver s, int variant) {
    if (!s) return fail(SFG_ERR_ARG, "null solver");
    if (variant < 0 || variant > 2) return fail(SFG_ERR_ARG, "unknown kernel variant %d", variant);
    if (variant > 1 && s->grid.dim == 3) return fail(SFG_ERR_ARG, "3-D grids have variants 0 (sweeps) and 1 (tiles)");
    // variant 2: the 22 x 22 tile (2-D), the whole-run cluster kernel (1-D)
    if (variant != s->variant && s->graph) {
        cudaGraphExecDestroy(s->graph);
        s->graph = nullptr;
    }
    s->variant = variant;
    return SFG_OK;
}

int sfg_get_kernel_variant(sfg_solver s, int* variant) {
    if (!s || !variant) return fail(SFG_ERR_ARG, "null argument");
    *variant = s->variant;
    return SFG_OK;
}

int sfg_get_counters(sfg_solver s, uint64_t* teno_cores, uint64_t* teno_cut) {
    if (!s) return fail(SFG_ERR_ARG, "null solver");
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    unsigned long long c[2];
    CUDA_TRY(cudaMemcpy(c, s->counters, sizeof c, cudaMemcpyDeviceToHost));
    if (teno_cores) *teno_cores = c[0];
    if (teno_cut) *teno_cut = c[1];
    return SFG_OK;
}

}  // extern "C"
