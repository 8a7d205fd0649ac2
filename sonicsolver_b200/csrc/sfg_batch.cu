// sfg_batch.cu -- many independent grids of uneven sizes and dimensions
// advanced together (sfg_batch_* in include/sonicsolver_b200.h).
//
// Device side:
//   * an instance table: per grid its GridView, state buffers (carved out of
//     one HBM slab), its own step clock (t, CFL dt, end time, step limit) and
//     status word -- every grid keeps its own CFL step, exactly as if it ran
//     alone;
//   * a work list of tiles (2-D: TX x TY nodes, 1-D: 511 nodes) covering the
//     solved nodes of every live instance, with its length in device memory;
//   * a step of four launches: the per-instance dt (the CFL minimum was
//     reduced by the previous step's last stage, per-instance 64-bit
//     atomicMin; a grid's first one when it joins), each stage as persistent
//     kernels, one block per SM slot, that take tiles from the list with an
//     atomic counter (the fused tile bodies of sfg_tile.cuh), then the
//     per-instance clock update.
// Every grid carries its own numerics (convection recipe, gamma, CFL,
// maxDeltaT), as every reference case directory selects its own TermRecipe.
// Grids of one recipe form a group: the work list holds the groups' tiles in
// contiguous ranges, and each stage runs one persistent kernel per group (the
// recipe's template instance), the groups' kernels on parallel branches so
// that one group's blocks fill the SMs that another's tail leaves idle.
// A grid may have frozen ends (a patch without a condition) and law ends
// (fixedValue / zeroGradient / symmetry laws per field) as a single-grid
// solver has them: the instance's device grid carries the extra end nodes,
// and a law kernel applies every law instance's laws at the points the
// single-grid solver does (step start, before each stage's RHS, after the
// last stage), with the same arithmetic (sfg_laws.cuh).
// Host side: the batch step is captured once as a CUDA graph of G steps.
// Adding or removing instances rewrites the table rows and the work list in
// device memory between graph launches, so the graph needs recapture only
// when a grid brings a recipe the batch has not run yet (continuous
// batching).
#include "../../include/sonicsolver_b200.h"
#include "sfg_laws.cuh"
#include "sfg_tile.cuh"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdarg>
#include <cstring>
#include <limits>
#include <map>
#include <string>
#include <vector>

namespace sfg {
void set_last_error(const char* msg);
cudaError_t launch_soa_to_aos(const GridView& g, const double* soa, double* aos, cudaStream_t st);
cudaError_t launch_aos_to_soa(const double* aos, double* soa, long long nodes, long long vs, cudaStream_t st);

struct BatchInst {
    GridView g;
    double *qn, *qa, *qb, *k;
    const LawView* law;  // law ends (device copy in the slab), or null
    Clock clock;
    unsigned flags;
    int live;  // slot in use
    int done;  // reached its end time / step limit or failed (set by finalize)
    int pad;
};

// A tile: 2-D, TX x TY nodes from (x0, y0); 1-D, y0 nodes (TILE1D, or
// TILE1D_SHORT once the batch has drained) from x0.
struct WorkItem {
    int inst, x0, y0, dim;
};

// A run of up to LAW_CHUNK face points of one law instance.
constexpr int LAW_CHUNK = 128;
struct LawItem {
    int inst, first, count, pad;
};

constexpr int kMaxGroups = 8;  // one per convection recipe the batch kernels provide
constexpr int kCounters = 8 + 4 * kMaxGroups;

struct BatchCtl {
    int n_items;
    int n_inst;
    int active;   // instances stepping in the current step (counted by finalize)
    int stepped;  // instances that stepped in the last completed step (set by commit)
    int n_law_items;
    int pad;
    // work stealing: [5] copy, [8 + 4 g + s] stage s of recipe group g
    int counters[kCounters];
    // tile range of group g in the work list: [2 g] first item, [2 g + 1] count
    int group_range[2 * kMaxGroups];
};

// ---------------------------------------------------------------- kernels

__device__ __forceinline__ int steal(int* counter, int* slot) {
    if (threadIdx.x == 0) *slot = atomicAdd(counter, 1);
    __syncthreads();
    const int item = *slot;
    __syncthreads();
    return item;
}

__device__ __forceinline__ StageView batch_stage_view(BatchInst& b, int stage, int time_id) {
    StageView sv{};
    sv.clock = &b.clock;
    sv.flags = &b.flags;
    sv.counters = nullptr;
    sv.time_id = time_id;
    sv.stage = stage;
    sv.q0 = b.qn;
    sv.r = nullptr;
    sv.k = b.k;
    sv.mode = MODE_FINAL;
    sv.require_active = 0;
    if (time_id == T_EULER) {
        sv.qs = b.qn;
        sv.qout = b.qa;
    } else if (time_id == T_SSPRK3) {
        const double base[3] = {0.0, 0.75, 1.0 / 3.0};
        const double inc[3] = {1.0, 0.25, 2.0 / 3.0};
        sv.base = base[stage];
        sv.inc = inc[stage];
        sv.qs = stage == 0 ? b.qn : (stage == 1 ? b.qa : b.qb);
        sv.qout = stage == 0 ? b.qa : (stage == 1 ? b.qb : b.qn);
    } else {
        const double inc[4] = {0.5, 0.5, 1.0, 0.0};
        sv.inc = inc[stage];
        sv.qs = stage == 0 ? b.qn : (stage == 1 ? b.qa : (stage == 2 ? b.qb : b.qa));
        sv.qout = stage == 0 ? b.qa : (stage == 1 ? b.qb : (stage == 2 ? b.qa : b.qn));
    }
    return sv;
}

// One stage over the tiles of recipe group `group` (the grids whose recipe is
// this instance's SCHEME and FLUX).
template <int SCHEME, int FLUX, bool F32, int TX, int TY>
__global__ void __launch_bounds__(TILE_THREADS, F32 ? 4 : 2)
    batch_stage_kernel(BatchInst* inst, const WorkItem* items, BatchCtl* ctl, int stage, int time_id, int group) {
    using Tt = typename std::conditional<F32, float, double>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Tt* smem = reinterpret_cast<Tt*>(smem_raw);
    __shared__ int slot;
    const int first = ctl->group_range[2 * group], n_items = ctl->group_range[2 * group + 1];
    for (;;) {
        const int it = steal(&ctl->counters[8 + 4 * group + stage], &slot);
        if (it >= n_items) break;
        const WorkItem w = items[first + it];
        BatchInst& b = inst[w.inst];
        if (!b.live || !b.clock.active) continue;  // uniform across the block
        StageView sv = batch_stage_view(b, stage, time_id);
        const bool last = stage == (time_id == T_EULER ? 0 : (time_id == T_SSPRK3 ? 2 : 3));
        if (last) sv.mode |= MODE_CFL;  // the step's result: reduce its CFL minimum here
        unsigned flags = 0, cut = 0, cores = 0;
        double sr = 0.0;
        if (w.dim == 2) {
            if constexpr (F32) tile2d_f32_body<SCHEME, FLUX, TX, TY>(b.g, sv, w.x0, w.y0, smem, flags, cut, cores, sr);
            else tile2d_body<SCHEME, FLUX, TX, TY>(b.g, sv, w.x0, w.y0, smem, flags, cut, cores, sr);
        } else if (w.y0 == TILE1D_SHORT) {
            tile1d_body<SCHEME, FLUX, Tt, TILE1D_SHORT>(b.g, sv, w.x0, smem, flags, cut, cores, sr);
        } else {
            tile1d_body<SCHEME, FLUX, Tt>(b.g, sv, w.x0, smem, flags, cut, cores, sr);
        }
        if (flags) atomicOr(&b.flags, flags);
        if (last) flush_cfl_block(b.g, &b.clock, sr);
        __syncthreads();  // shared arrays are reused by the next tile
    }
}

// The boundary laws of every stepping law instance, where the single-grid
// solver applies them: phase 0 at the step's start (FlowStepPrepare, on qn),
// phase 1 before stage `stage` reads its input (prepareBoundaryState; the
// previous application's values sit in the previous stage's input), phase 2
// on the last stage's output (FlowStepCommit).
__global__ void __launch_bounds__(LAW_CHUNK)
    batch_law_kernel(BatchInst* inst, const LawItem* items, BatchCtl* ctl, int phase, int stage, int time_id) {
    const int n = ctl->n_law_items;
    for (int k = blockIdx.x; k < n; k += gridDim.x) {
        const LawItem w = items[k];
        BatchInst& b = inst[w.inst];
        if (!b.live || !b.clock.active || !b.law || (int)threadIdx.x >= w.count) continue;
        const double* old = b.qn;
        double* q = b.qn;
        if (phase == 1) {
            q = const_cast<double*>(batch_stage_view(b, stage, time_id).qs);
            if (stage > 0) old = batch_stage_view(b, stage - 1, time_id).qs;
        } else if (phase == 2) {
            const StageView last = batch_stage_view(b, stage, time_id);
            q = last.qout;
            old = last.qs;
        }
        law_fill_point(b.g, *b.law, old, q, (long long)w.first + threadIdx.x, &b.flags);
    }
}

// CFL minimum of a grid's uploaded state (RusanovEOS::deltaT), once when it
// joins the batch; from then on each step's last stage reduces the new
// state's minimum (MODE_CFL), so the step itself has no CFL pass.
__global__ void __launch_bounds__(TILE_THREADS) batch_initial_cfl_kernel(BatchInst* inst, int idx) {
    BatchInst& b = inst[idx];
    const GridView& g = b.g;
    const int sx = g.hi[0] - g.lo[0], sy = g.hi[1] - g.lo[1];
    const long long count = (long long)sx * sy;
    double best = 0.0;
    unsigned fl = 0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < count;
         t += (long long)gridDim.x * blockDim.x) {
        const int i = g.lo[0] + (int)(t % sx), j = g.lo[1] + (int)(t / sx);
        const long long node = (long long)j * g.n[0] + i;
        const double* q = b.qn;
        const double qq[5] = {q[node], q[g.vs + node], q[2 * g.vs + node], q[3 * g.vs + node], q[4 * g.vs + node]};
        const double sr = cfl_rate(g, qq);
        if (!(sr > 0.0) || !isfinite(sr)) fl |= FLAG_NONFINITE;
        best = fmax(best, sr);
    }
    flush_cfl_block(g, &b.clock, best);
    if (fl) atomicOr(&b.flags, fl);
}

// FlowDtCompute + Time::Driver clipping per instance (one thread each).
__global__ void batch_finalize_kernel(BatchInst* inst, BatchCtl* ctl) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ctl->n_inst) return;
    BatchInst& b = inst[i];
    if (!b.live || b.done) return;
    Clock* c = &b.clock;
    const double eps = 2.220446049250313e-16;
    const double remaining = c->t_end - c->t;
    double scale = fmax(fabs(c->t), fabs(c->t_end));
    scale = scale < 1.0 ? 1.0 : scale;
    if (b.flags || !(remaining > 64.0 * eps * scale) || c->steps >= c->max_steps) {
        c->active = 0;
        c->dt = 0.0;
        b.done = 1;
        return;
    }
    double limit = remaining;
    if (c->write_interval > 0.0 && c->next_out - c->t < limit) limit = c->next_out - c->t;
    double dt = __longlong_as_double((long long)c->dt_bits);
    if (c->max_dt < dt) dt = c->max_dt;
    if (limit < dt) dt = limit;
    c->dt = dt;
    c->active = 1;
    c->dt_bits = 0x7FEFFFFFFFFFFFFFull;  // consumed: re-armed for the last stage's reduction
    c->dt_ready = 0;
    atomicAdd(&ctl->active, 1);
}

// Euler: the stage wrote qa; the committed state lives in qn.
template <int TX, int TY>
__global__ void __launch_bounds__(TILE_THREADS) batch_copy_kernel(BatchInst* inst, const WorkItem* items, BatchCtl* ctl) {
    __shared__ int slot;
    const int n_items = ctl->n_items;
    for (;;) {
        const int it = steal(&ctl->counters[5], &slot);
        if (it >= n_items) break;
        const WorkItem w = items[it];
        BatchInst& b = inst[w.inst];
        if (!b.live || !b.clock.active) continue;
        const int cnt = w.dim == 2 ? TX * TY : w.y0;
        for (int t = threadIdx.x; t < cnt; t += blockDim.x) {
            const int i = w.dim == 2 ? w.x0 + t % TX : w.x0 + t;
            const int j = w.dim == 2 ? w.y0 + t / TX : 0;
            if (i >= b.g.hi[0] || (w.dim == 2 && j >= b.g.hi[1])) continue;
            const long long node = (long long)j * b.g.n[0] + i;
            for (int v = 0; v < 5; ++v) b.qn[v * b.g.vs + node] = b.qa[v * b.g.vs + node];
        }
    }
}

// TimeCommit per instance; re-arms the per-step counters (one grid).
__global__ void batch_commit_kernel(BatchInst* inst, BatchCtl* ctl) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < ctl->n_inst) {
        BatchInst& b = inst[i];
        if (b.live) {
            Clock* c = &b.clock;
            if (c->active) {
                c->t += c->dt;
                c->steps += 1;
                double sc = fabs(c->t);
                sc = sc < 1.0 ? 1.0 : sc;
                if (c->write_interval > 0.0 && c->t >= c->next_out - 1.0e-11 * sc) c->next_out += c->write_interval;
            }
            c->dt_ready = c->active ? 1 : 0;  // the last stage reduced the new state's CFL minimum
        }
    }
    if (blockIdx.x == 0) {
        for (int c = threadIdx.x; c < kCounters; c += blockDim.x) ctl->counters[c] = 0;
        if (threadIdx.x == 0) {  // the next step's finalize counts afresh
            ctl->stepped = ctl->active;
            ctl->active = 0;
        }
    }
}

}  // namespace sfg

using namespace sfg;

// ---------------------------------------------------------------- host

namespace {

int bfail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    set_last_error(buf);
    return code;
}

#define BCUDA(expr)                                                                              \
    do {                                                                                         \
        cudaError_t e_ = (expr);                                                                 \
        if (e_ != cudaSuccess) return bfail(SFG_ERR_CUDA, "%s: %s", #expr, cudaGetErrorString(e_)); \
    } while (0)

struct RecipeParts {
    int id, scheme, flux;
};
const RecipeParts kBatchRecipes[] = {
    {SFG_RECIPE_WENO3_RUSANOV, WENO3, RUSANOV}, {SFG_RECIPE_WENO3_ROE, WENO3, ROE},
    {SFG_RECIPE_WENO5_RUSANOV, WENO5, RUSANOV}, {SFG_RECIPE_WENO5_ROE, WENO5, ROE},
    {SFG_RECIPE_TENO5_RUSANOV, TENO5, RUSANOV}, {SFG_RECIPE_TENO5_ROE, TENO5, ROE},
    {SFG_RECIPE_WENO7_RUSANOV, WENO7, RUSANOV}, {SFG_RECIPE_WENO7_ROE, WENO7, ROE}};

using StageKernel = void (*)(BatchInst*, const WorkItem*, BatchCtl*, int, int, int);
using ItemKernel = void (*)(BatchInst*, const WorkItem*, BatchCtl*);

template <int TX, int TY, bool F32>
StageKernel pick_stage(int scheme, int flux) {
#define SFG_PICK(S)                                                                              \
    if (scheme == S) return flux == RUSANOV ? batch_stage_kernel<S, RUSANOV, F32, TX, TY>        \
                                            : batch_stage_kernel<S, ROE, F32, TX, TY>;
    SFG_PICK(WENO5)
    SFG_PICK(TENO5)
    SFG_PICK(WENO3)
    SFG_PICK(WENO7)
#undef SFG_PICK
    return nullptr;
}

template <int TX, int TY>
size_t stage_smem(int scheme, bool f32) {
    size_t e2 = 0, e1 = 0;
    switch (scheme) {
    case WENO3: e2 = TileShape<WENO3, TX, TY>::ELEMS; e1 = Tile1Shape<WENO3>::ELEMS; break;
    case WENO5: e2 = TileShape<WENO5, TX, TY>::ELEMS; e1 = Tile1Shape<WENO5>::ELEMS; break;
    case TENO5: e2 = TileShape<TENO5, TX, TY>::ELEMS; e1 = Tile1Shape<TENO5>::ELEMS; break;
    default: e2 = TileShape<WENO7, TX, TY>::ELEMS; e1 = Tile1Shape<WENO7>::ELEMS; break;
    }
    return std::max(e2, e1) * (f32 ? sizeof(float) : sizeof(double));
}

int stage_count_of(int time_id) { return time_id == T_EULER ? 1 : (time_id == T_SSPRK3 ? 3 : 4); }

const double kInfB = std::numeric_limits<double>::infinity();

}  // namespace

// The grids of one convection recipe: their stage kernel, its launch shape,
// and the stream its branch of a stage runs on (group 0: the batch's stream).
struct RecipeGroup {
    const RecipeParts* recipe = nullptr;
    StageKernel stage_k = nullptr;
    size_t smem = 0;
    int grid = 0;
    cudaStream_t side = nullptr;
    cudaEvent_t joined = nullptr;
};

struct sfg_batch_s {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    sfg_numerics_desc num{};
    const RecipeParts* recipe = nullptr;  // the default recipe (group 0)
    std::vector<RecipeGroup> groups;
    std::vector<int> inst_group;          // per slot
    cudaEvent_t fork = nullptr;
    int variant = 1;  // 1: 32 x 15 tiles, 2: 22 x 22
    int tx = 32, ty = 15;
    int max_inst = 0;
    // HBM slab for instance state, first-fit allocator over it
    char* slab = nullptr;
    size_t budget = 0, used = 0;
    std::map<size_t, size_t> free_blocks;  // offset -> size
    // tables
    BatchInst* d_inst = nullptr;
    std::vector<BatchInst> h_inst;
    std::vector<size_t> inst_offset, inst_bytes;
    WorkItem* d_items = nullptr;
    size_t items_cap = 0;
    std::vector<WorkItem> h_items;
    // per slot: the caller's grid and the device grid's offset (extra end
    // nodes of frozen and law ends), its law view (count 0: none)
    std::vector<sfg_grid_desc> inst_pub;
    std::vector<std::array<int, 3>> inst_off;
    std::vector<LawView> inst_law;
    bool has_laws = false;  // a law instance was added: the step graph has the law launches
    LawItem* d_law_items = nullptr;
    size_t law_items_cap = 0;
    std::vector<LawItem> h_law_items;
    int law_grid = 0;
    BatchCtl* d_ctl = nullptr;
    BatchCtl* h_ctl = nullptr;  // pinned
    double* staging = nullptr;
    size_t staging_cap = 0;
    // kernels and graph
    ItemKernel copy_k = nullptr;
    int grid_items = 0;
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0;
    long long batch_steps = 0;
};

namespace {

// Stage kernel of one recipe group for the batch's tile shape and precision.
int bind_group(sfg_batch_s* b, RecipeGroup& grp) {
    const bool f32 = b->num.precision == SFG_PREC_FP32_FLUX;
    const int scheme = grp.recipe->scheme, flux = grp.recipe->flux;
    if (b->variant == 1) {
        grp.stage_k = f32 ? pick_stage<32, 15, true>(scheme, flux) : pick_stage<32, 15, false>(scheme, flux);
        grp.smem = stage_smem<32, 15>(scheme, f32);
    } else {
        grp.stage_k = f32 ? pick_stage<22, 22, true>(scheme, flux) : pick_stage<22, 22, false>(scheme, flux);
        grp.smem = stage_smem<22, 22>(scheme, f32);
    }
    if (!grp.stage_k) return bfail(SFG_ERR_ARG, "no batched stage kernel for recipe %d", grp.recipe->id);
    BCUDA(cudaFuncSetAttribute(grp.stage_k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)grp.smem));
    int sms = 0, per_sm = 0;
    BCUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device));
    BCUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, grp.stage_k, TILE_THREADS, grp.smem));
    if (per_sm < 1) return bfail(SFG_ERR_CUDA, "batched stage kernel does not fit an SM");
    grp.grid = sms * per_sm;
    return SFG_OK;
}

int bind_kernels(sfg_batch_s* b) {
    if (b->variant == 1) {
        b->copy_k = batch_copy_kernel<32, 15>;
        b->tx = 32;
        b->ty = 15;
    } else {
        b->copy_k = batch_copy_kernel<22, 22>;
        b->tx = 22;
        b->ty = 22;
    }
    for (auto& grp : b->groups) {
        int rc = bind_group(b, grp);
        if (rc) return rc;
    }
    int sms = 0;
    BCUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device));
    b->grid_items = sms * 4;
    b->law_grid = sms * 8;
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    return SFG_OK;
}

// Group index of a recipe; a recipe the batch has not run yet opens a group
// (its kernel bound, a stream for its branch), which the next captured graph
// includes.
int group_of(sfg_batch_s* b, const RecipeParts* rp, int* out) {
    for (int g = 0; g < (int)b->groups.size(); ++g)
        if (b->groups[g].recipe == rp) {
            *out = g;
            return SFG_OK;
        }
    if ((int)b->groups.size() >= kMaxGroups) return bfail(SFG_ERR_ARG, "too many recipes in one batch");
    RecipeGroup grp;
    grp.recipe = rp;
    int rc = bind_group(b, grp);
    if (rc) return rc;
    if (!b->groups.empty()) {
        BCUDA(cudaStreamCreateWithFlags(&grp.side, cudaStreamNonBlocking));
        if (cudaEventCreateWithFlags(&grp.joined, cudaEventDisableTiming) != cudaSuccess) {
            cudaStreamDestroy(grp.side);
            return bfail(SFG_ERR_CUDA, "event creation failed");
        }
    }
    b->groups.push_back(grp);
    if (b->graph) {  // the graph has no branch for the new group
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    *out = (int)b->groups.size() - 1;
    return SFG_OK;
}

int slab_alloc(sfg_batch_s* b, size_t bytes, size_t* off) {
    bytes = (bytes + 255) / 256 * 256;
    for (auto it = b->free_blocks.begin(); it != b->free_blocks.end(); ++it) {
        if (it->second >= bytes) {
            *off = it->first;
            const size_t rest = it->second - bytes;
            const size_t roff = it->first + bytes;
            b->free_blocks.erase(it);
            if (rest) b->free_blocks[roff] = rest;
            b->used += bytes;
            return SFG_OK;
        }
    }
    return bfail(SFG_ERR_BUDGET, "HBM budget exhausted: %zu bytes requested, %zu of %zu in use", bytes, b->used,
                 b->budget);
}

void slab_free(sfg_batch_s* b, size_t off, size_t bytes) {
    bytes = (bytes + 255) / 256 * 256;
    b->used -= bytes;
    auto it = b->free_blocks.emplace(off, bytes).first;
    auto next = std::next(it);
    if (next != b->free_blocks.end() && it->first + it->second == next->first) {
        it->second += next->second;
        b->free_blocks.erase(next);
    }
    if (it != b->free_blocks.begin()) {
        auto prev = std::prev(it);
        if (prev->first + prev->second == it->first) {
            prev->second += it->second;
            b->free_blocks.erase(it);
        }
    }
}

// Rebuilds the tile list of all live instances and publishes it (and the
// instance count) to device memory.
int publish_items(sfg_batch_s* b) {
    b->h_items.clear();
    // 1-D tiles of one face round once the live tiles no longer fill the
    // SMs: a drained batch's last grids then take half the time per stage
    long long long_tiles = 0;
    for (int i = 0; i < (int)b->h_inst.size(); ++i) {
        const BatchInst& r = b->h_inst[i];
        if (!r.live || r.done) continue;
        const GridView& g = r.g;
        long_tiles += g.dim == 1 ? (g.hi[0] - g.lo[0] + TILE1D - 1) / TILE1D
                                 : (long long)((g.hi[0] - g.lo[0] + b->tx - 1) / b->tx) *
                                       ((g.hi[1] - g.lo[1] + b->ty - 1) / b->ty);
    }
    const int t1 = long_tiles < b->grid_items ? TILE1D_SHORT : TILE1D;
    for (int grp = 0; grp < kMaxGroups; ++grp) {
        const int first = (int)b->h_items.size();
        for (int i = 0; grp < (int)b->groups.size() && i < (int)b->h_inst.size(); ++i) {
            const BatchInst& r = b->h_inst[i];
            if (!r.live || r.done || b->inst_group[i] != grp) continue;
            const GridView& g = r.g;
            if (g.dim == 1) {
                for (int x = g.lo[0]; x < g.hi[0]; x += t1) b->h_items.push_back({i, x, t1, 1});
            } else {
                for (int y = g.lo[1]; y < g.hi[1]; y += b->ty)
                    for (int x = g.lo[0]; x < g.hi[0]; x += b->tx) b->h_items.push_back({i, x, y, 2});
            }
        }
        b->h_ctl->group_range[2 * grp] = first;
        b->h_ctl->group_range[2 * grp + 1] = (int)b->h_items.size() - first;
    }
    if (b->h_items.size() > b->items_cap) {
        size_t cap = std::max<size_t>(b->h_items.size() * 2, 1024);
        if (b->d_items) cudaFree(b->d_items);
        b->d_items = nullptr;
        BCUDA(cudaMalloc((void**)&b->d_items, cap * sizeof(WorkItem)));
        b->items_cap = cap;
        if (b->graph) {  // the graph holds the old list address
            cudaGraphExecDestroy(b->graph);
            b->graph = nullptr;
        }
    }
    if (!b->h_items.empty())
        BCUDA(cudaMemcpyAsync(b->d_items, b->h_items.data(), b->h_items.size() * sizeof(WorkItem),
                              cudaMemcpyHostToDevice, b->stream));
    // law points of the live law instances, in runs of LAW_CHUNK
    b->h_law_items.clear();
    for (int i = 0; i < (int)b->h_inst.size(); ++i) {
        const BatchInst& r = b->h_inst[i];
        if (!r.live || r.done || !r.law) continue;
        const LawView& lv = b->inst_law[i];
        const int pts = (int)lv.start[lv.count];
        for (int f = 0; f < pts; f += LAW_CHUNK) b->h_law_items.push_back({i, f, std::min(LAW_CHUNK, pts - f), 0});
    }
    if (b->h_law_items.size() > b->law_items_cap) {
        size_t cap = std::max<size_t>(b->h_law_items.size() * 2, 256);
        if (b->d_law_items) cudaFree(b->d_law_items);
        b->d_law_items = nullptr;
        BCUDA(cudaMalloc((void**)&b->d_law_items, cap * sizeof(LawItem)));
        b->law_items_cap = cap;
        if (b->graph) {  // the graph holds the old list address
            cudaGraphExecDestroy(b->graph);
            b->graph = nullptr;
        }
    }
    if (!b->h_law_items.empty())
        BCUDA(cudaMemcpyAsync(b->d_law_items, b->h_law_items.data(), b->h_law_items.size() * sizeof(LawItem),
                              cudaMemcpyHostToDevice, b->stream));
    b->h_ctl->n_law_items = (int)b->h_law_items.size();
    BCUDA(cudaMemcpyAsync(&b->d_ctl->n_law_items, &b->h_ctl->n_law_items, sizeof(int), cudaMemcpyHostToDevice,
                          b->stream));
    b->h_ctl->n_items = (int)b->h_items.size();
    b->h_ctl->n_inst = (int)b->h_inst.size();
    BCUDA(cudaMemcpyAsync(&b->d_ctl->n_items, &b->h_ctl->n_items, 2 * sizeof(int), cudaMemcpyHostToDevice, b->stream));
    BCUDA(cudaMemcpyAsync(b->d_ctl->group_range, b->h_ctl->group_range, sizeof b->h_ctl->group_range,
                          cudaMemcpyHostToDevice, b->stream));
    BCUDA(cudaStreamSynchronize(b->stream));
    return SFG_OK;
}

int enqueue_batch_step(sfg_batch_s* b) {
    const int ni = std::max<int>(1, b->max_inst);
    batch_finalize_kernel<<<(ni + 127) / 128, 128, 0, b->stream>>>(b->d_inst, b->d_ctl);
    const int ns = stage_count_of(b->num.time_recipe);
    const int ng = (int)b->groups.size();
    auto laws = [&](int phase, int stage) {
        batch_law_kernel<<<b->law_grid, LAW_CHUNK, 0, b->stream>>>(b->d_inst, b->d_law_items, b->d_ctl, phase, stage,
                                                                 b->num.time_recipe);
    };
    if (b->has_laws) laws(0, 0);  // FlowStepPrepare
    for (int s = 0; s < ns; ++s) {
        if (b->has_laws) laws(1, s);  // the stage input's boundary state
        // group 0 on the batch's stream, every other group on a branch
        // forked from it and joined back before the next stage
        if (ng > 1) BCUDA(cudaEventRecord(b->fork, b->stream));
        for (int g = 0; g < ng; ++g) {
            const RecipeGroup& grp = b->groups[g];
            cudaStream_t st = g == 0 ? b->stream : grp.side;
            if (g > 0) BCUDA(cudaStreamWaitEvent(st, b->fork, 0));
            grp.stage_k<<<grp.grid, TILE_THREADS, grp.smem, st>>>(b->d_inst, b->d_items, b->d_ctl, s,
                                                                   b->num.time_recipe, g);
            if (g > 0) BCUDA(cudaEventRecord(grp.joined, st));
        }
        for (int g = 1; g < ng; ++g) BCUDA(cudaStreamWaitEvent(b->stream, b->groups[g].joined, 0));
    }
    if (b->has_laws) laws(2, ns - 1);  // FlowStepCommit on the last stage's output
    if (b->num.time_recipe == T_EULER) b->copy_k<<<b->grid_items, TILE_THREADS, 0, b->stream>>>(b->d_inst, b->d_items, b->d_ctl);
    batch_commit_kernel<<<(ni + 127) / 128, 128, 0, b->stream>>>(b->d_inst, b->d_ctl);
    BCUDA(cudaGetLastError());
    return SFG_OK;
}

// Checks a grid's own numerics against the batch (same time recipe and
// precision; a recipe with a batched kernel; gamma, CFL and maxDeltaT as
// sfg_create accepts them) and returns its recipe.
int instance_numerics(const sfg_batch_s* b, const sfg_numerics_desc* n, const RecipeParts** rp) {
    *rp = nullptr;
    for (const auto& r : kBatchRecipes)
        if (r.id == n->recipe) *rp = &r;
    if (!*rp) return bfail(SFG_ERR_ARG, "convection recipe %d is not provided on the GPU", n->recipe);
    if (n->time_recipe != b->num.time_recipe) return bfail(SFG_ERR_ARG, "a batch runs one time recipe");
    if (n->precision != b->num.precision) return bfail(SFG_ERR_ARG, "a batch runs one precision mode");
    if (!(n->gamma > 1.0) || !std::isfinite(n->gamma)) return bfail(SFG_ERR_ARG, "gamma must be > 1");
    if (!(n->cfl > 0.0) || !std::isfinite(n->cfl)) return bfail(SFG_ERR_ARG, "CFL must be finite and > 0");
    if (n->max_dt != n->max_dt) return bfail(SFG_ERR_ARG, "maxDeltaT is NaN");
    return SFG_OK;
}

// Device view of a grid: one extra node at every frozen and law end (it
// holds the frozen ghost value, or the law's ghost value), as the
// single-grid solver lays its grid out; off_lo: the offset of the caller's
// node 0 on each axis.  *nodes: the device grid's node count.
int batch_grid_view(const sfg_grid_desc* d, const sfg_numerics_desc* n, int reach, GridView* out, long long* nodes,
                    int off_lo[3]) {
    if (!d) return bfail(SFG_ERR_ARG, "null grid");
    if (d->dim < 1 || d->dim > 2) return bfail(SFG_ERR_ARG, "batched grids are 1-D or 2-D (got %d)", d->dim);
    GridView g{};
    g.dim = d->dim;
    auto extra_end = [](int bk) { return bk == SFG_BC_FROZEN || bk == SFG_BC_LAW; };
    for (int a = 0; a < 3; ++a) {
        off_lo[a] = 0;
        if (!(d->h[a] > 0.0)) return bfail(SFG_ERR_ARG, "h[%d] must be > 0", a);
        g.n[a] = d->n[a];
        if (a >= d->dim) {
            if (d->n[a] != 1) return bfail(SFG_ERR_ARG, "inactive axis %d must have 1 node", a);
            g.lo[a] = 0;
            g.hi[a] = 1;
            continue;
        }
        const bool plo = d->bc_lo[a] == SFG_BC_PERIODIC, phi = d->bc_hi[a] == SFG_BC_PERIODIC;
        if (plo != phi) return bfail(SFG_ERR_ARG, "axis %d: periodic must be set on both ends", a);
        for (int bk : {d->bc_lo[a], d->bc_hi[a]})
            if (bk != SFG_BC_TRANSMISSIVE && bk != SFG_BC_PERIODIC && bk != SFG_BC_FROZEN && bk != SFG_BC_LAW)
                return bfail(SFG_ERR_ARG, "unknown boundary kind");
        off_lo[a] = extra_end(d->bc_lo[a]) ? 1 : 0;
        const int nd = d->n[a] + off_lo[a] + (extra_end(d->bc_hi[a]) ? 1 : 0);
        if (plo ? d->n[a] < reach + 1 : nd < 3) return bfail(SFG_ERR_ARG, "axis %d has too few nodes", a);
        g.n[a] = nd;
        // a law end reads like a frozen one: ghosts clamp to its extra node
        g.bc_lo[a] = d->bc_lo[a] == SFG_BC_LAW ? BC_FROZEN : d->bc_lo[a];
        g.bc_hi[a] = d->bc_hi[a] == SFG_BC_LAW ? BC_FROZEN : d->bc_hi[a];
        // transmissive and law boundary nodes and extra nodes are not advanced
        g.lo[a] = plo ? 0 : (d->bc_lo[a] == SFG_BC_LAW ? 2 : 1);
        g.hi[a] = plo ? nd : (d->bc_hi[a] == SFG_BC_LAW ? nd - 2 : nd - 1);
        if (g.hi[a] <= g.lo[a]) return bfail(SFG_ERR_ARG, "axis %d has no solved node", a);
    }
    const double hx = d->h[0], hy = d->h[1], hz = d->h[2];
    g.jac = 1.0 / (hx * hy * hz);
    g.metric[0] = (hy * hz) * g.jac;
    g.metric[1] = (hx * hz) * g.jac;
    g.metric[2] = (hx * hy) * g.jac;
    for (int a = 0; a < 3; ++a) g.area[a] = 0.5 * (g.metric[a] / g.jac + g.metric[a] / g.jac);
    g.gamma = n->gamma;
    for (int a = 0; a < 3; ++a) g.h[a] = d->h[a];
    g.cfl = n->cfl;
    *nodes = (long long)g.n[0] * g.n[1] * g.n[2];
    g.vs = (*nodes + 31) / 32 * 32;
    *out = g;
    return SFG_OK;
}

bool has_extra_nodes(const GridView& g, const sfg_grid_desc& pub) {
    return g.n[0] != pub.n[0] || g.n[1] != pub.n[1] || g.n[2] != pub.n[2];
}

// Caller node layout -> device layout (AoS): an extra end node takes its
// boundary node's value (the reference fills ghosts by clamping to the
// interior, SF_mesh.cpp:544), as sfg_upload does.
void to_device_layout(const sfg_grid_desc& pub, const GridView& g, const int off[3], const double* in,
                      std::vector<double>& out) {
    out.resize(5 * (size_t)g.n[0] * g.n[1] * g.n[2]);
    for (int k = 0; k < g.n[2]; ++k)
        for (int j = 0; j < g.n[1]; ++j)
            for (int i = 0; i < g.n[0]; ++i) {
                int c[3] = {i - off[0], j - off[1], k - off[2]};
                for (int a = 0; a < 3; ++a) c[a] = std::min(std::max(c[a], 0), pub.n[a] - 1);
                std::memcpy(&out[(((size_t)k * g.n[1] + j) * g.n[0] + i) * 5],
                            in + (((size_t)c[2] * pub.n[1] + c[1]) * pub.n[0] + c[0]) * 5, 5 * sizeof(double));
            }
}

// Device layout (AoS) -> caller node layout (drops the extra end nodes).
void to_caller_layout(const sfg_grid_desc& pub, const GridView& g, const int off[3], const double* in, double* out) {
    for (int k = 0; k < pub.n[2]; ++k)
        for (int j = 0; j < pub.n[1]; ++j)
            for (int i = 0; i < pub.n[0]; ++i)
                std::memcpy(out + (((size_t)k * pub.n[1] + j) * pub.n[0] + i) * 5,
                            in + (((size_t)(k + off[2]) * g.n[1] + (j + off[1])) * g.n[0] + (i + off[0])) * 5,
                            5 * sizeof(double));
}

size_t align256(size_t x) { return (x + 255) / 256 * 256; }

// Face points of a grid's law ends (over the solved range of the other axes).
long long law_points(const sfg_grid_desc& pub, const GridView& g) {
    long long pts = 0;
    for (int a = 0; a < pub.dim; ++a)
        for (int end = 0; end < 2; ++end) {
            if ((end ? pub.bc_hi[a] : pub.bc_lo[a]) != SFG_BC_LAW) continue;
            long long p = 1;
            for (int d = 0; d < 3; ++d)
                if (d != a) p *= g.hi[d] - g.lo[d];
            pts += p;
        }
    return pts;
}

// Slab bytes of one instance: its state buffers, and for law ends the law
// view and the state-cache codes.
size_t instance_slab_bytes(const sfg_batch_s* b, const sfg_grid_desc& pub, const GridView& g) {
    const size_t per = align256(sizeof(double) * 5 * (size_t)g.vs);
    const int bufs = b->num.time_recipe == T_RK4 ? 4 : 3;
    const long long pts = law_points(pub, g);
    return per * bufs + (pts > 0 ? align256(sizeof(LawView)) + align256((size_t)pts) : 0);
}

}  // namespace

namespace sfg {
// A request's own numerics, checked at submit before it queues (sfg_server.cu).
int batch_check_numerics(sfg_batch b, const sfg_numerics_desc* n) {
    const RecipeParts* rp = nullptr;
    return instance_numerics(b, n, &rp);
}
}  // namespace sfg

extern "C" {

int sfg_batch_create(const sfg_numerics_desc* numerics, size_t hbm_budget_bytes, int max_instances, void* stream,
                     sfg_batch* out) {
    if (!numerics || !out) return bfail(SFG_ERR_ARG, "null argument");
    *out = nullptr;
    const RecipeParts* rp = nullptr;
    for (const auto& r : kBatchRecipes)
        if (r.id == numerics->recipe) rp = &r;
    if (!rp) return bfail(SFG_ERR_ARG, "convection recipe %d is not provided on the GPU", numerics->recipe);
    if (numerics->time_recipe < 0 || numerics->time_recipe > 2) return bfail(SFG_ERR_ARG, "unknown time recipe");
    if (numerics->precision != SFG_PREC_FP64 && numerics->precision != SFG_PREC_FP32_FLUX)
        return bfail(SFG_ERR_ARG, "unknown precision");
    if (!(numerics->gamma > 1.0) || !(numerics->cfl > 0.0)) return bfail(SFG_ERR_ARG, "gamma > 1 and CFL > 0 required");
    if (max_instances < 1 || max_instances > (1 << 20)) return bfail(SFG_ERR_ARG, "max_instances out of range");
    if (hbm_budget_bytes < (1u << 20)) return bfail(SFG_ERR_ARG, "HBM budget below 1 MiB");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return bfail(SFG_ERR_CUDA, "no CUDA device: the B200 provider has no CPU fallback");
    auto* b = new sfg_batch_s;
    b->num = *numerics;
    if (!(b->num.max_dt > 0.0)) b->num.max_dt = kInfB;
    b->recipe = rp;
    b->max_inst = max_instances;
    cudaGetDevice(&b->device);
    auto cleanup = [&](int code) {
        sfg_batch_destroy(b);
        return code;
    };
    if (stream) {
        b->stream = (cudaStream_t)stream;
    } else {
        if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess)
            return cleanup(bfail(SFG_ERR_CUDA, "stream creation failed"));
        b->own_stream = true;
    }
    b->budget = hbm_budget_bytes / 256 * 256;
    if (cudaMalloc((void**)&b->slab, b->budget) != cudaSuccess)
        return cleanup(bfail(SFG_ERR_NOMEM, "cannot reserve the HBM budget of %zu bytes", b->budget));
    b->free_blocks[0] = b->budget;
    if (cudaMalloc((void**)&b->d_inst, sizeof(BatchInst) * (size_t)max_instances) != cudaSuccess ||
        cudaMalloc((void**)&b->d_ctl, sizeof(BatchCtl)) != cudaSuccess ||
        cudaMallocHost((void**)&b->h_ctl, sizeof(BatchCtl)) != cudaSuccess)
        return cleanup(bfail(SFG_ERR_NOMEM, "device allocation failed"));
    cudaMemsetAsync(b->d_inst, 0, sizeof(BatchInst) * (size_t)max_instances, b->stream);
    cudaMemsetAsync(b->d_ctl, 0, sizeof(BatchCtl), b->stream);
    std::memset(b->h_ctl, 0, sizeof(BatchCtl));
    if (cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess)
        return cleanup(bfail(SFG_ERR_CUDA, "event creation failed"));
    int rc = bind_kernels(b);
    if (rc) return cleanup(rc);
    int g0 = 0;
    rc = group_of(b, rp, &g0);  // the default recipe is group 0
    if (rc) return cleanup(rc);
    rc = publish_items(b);
    if (rc) return cleanup(rc);
    *out = b;
    return SFG_OK;
}

int sfg_batch_destroy(sfg_batch b) {
    if (!b) return SFG_OK;
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    if (b->slab) cudaFree(b->slab);
    if (b->d_inst) cudaFree(b->d_inst);
    if (b->d_items) cudaFree(b->d_items);
    if (b->d_law_items) cudaFree(b->d_law_items);
    if (b->d_ctl) cudaFree(b->d_ctl);
    if (b->staging) cudaFree(b->staging);
    if (b->h_ctl) cudaFreeHost(b->h_ctl);
    for (auto& grp : b->groups) {
        if (grp.side) cudaStreamDestroy(grp.side);
        if (grp.joined) cudaEventDestroy(grp.joined);
    }
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return SFG_OK;
}

int sfg_batch_instance_bytes(sfg_batch b, const sfg_grid_desc* grid, size_t* bytes) {
    if (!b || !grid || !bytes) return bfail(SFG_ERR_ARG, "null argument");
    GridView g;
    long long nodes = 0;
    int off[3];
    const int reach = b->recipe->scheme == WENO3 ? 2 : (b->recipe->scheme == WENO7 ? 4 : 3);
    int rc = batch_grid_view(grid, &b->num, reach, &g, &nodes, off);
    if (rc) return rc;
    *bytes = instance_slab_bytes(b, *grid, g);
    return SFG_OK;
}

int sfg_batch_add(sfg_batch b, const sfg_grid_desc* grid, const double* host_nodes_aos, double t_end,
                  int64_t max_steps, int* slot) {
    return sfg_batch_add_laws(b, grid, nullptr, nullptr, host_nodes_aos, t_end, max_steps, slot);
}

int sfg_batch_add_ex(sfg_batch b, const sfg_grid_desc* grid, const sfg_numerics_desc* numerics,
                     const double* host_nodes_aos, double t_end, int64_t max_steps, int* slot) {
    return sfg_batch_add_laws(b, grid, numerics, nullptr, host_nodes_aos, t_end, max_steps, slot);
}

int sfg_batch_add_laws(sfg_batch b, const sfg_grid_desc* grid, const sfg_numerics_desc* numerics,
                       const sfg_boundary_law* laws, const double* host_nodes_aos, double t_end, int64_t max_steps,
                       int* slot) {
    sfg::NvtxRange nvtx_("sfg_batch_add");
    if (!b || !grid || !host_nodes_aos || !slot) return bfail(SFG_ERR_ARG, "null argument");
    const sfg_numerics_desc& num = numerics ? *numerics : b->num;
    const RecipeParts* rp = nullptr;
    int rc = instance_numerics(b, &num, &rp);
    if (rc) return rc;
    GridView g;
    long long nodes = 0;
    int off[3];
    const int reach = rp->scheme == WENO3 ? 2 : (rp->scheme == WENO7 ? 4 : 3);
    rc = batch_grid_view(grid, &num, reach, &g, &nodes, off);
    if (rc) return rc;
    // law ends: every one needs its laws
    const long long pts = law_points(*grid, g);
    LawView lv{};
    std::vector<unsigned char> codes;
    if (pts > 0) {
        if (!laws) return bfail(SFG_ERR_ARG, "a grid with SFG_BC_LAW ends needs its laws (sfg_batch_add_laws)");
        for (int a = 0; a < grid->dim; ++a)
            for (int end = 0; end < 2; ++end)
                if ((end ? grid->bc_hi[a] : grid->bc_lo[a]) == SFG_BC_LAW)
                    if (const char* why = law_problem(laws[2 * a + end]))
                        return bfail(SFG_ERR_ARG, "axis %d end %d: %s", a, end, why);
        grid_law_view(*grid, g, off, laws, reach, lv, codes);
    }
    const bool extra = has_extra_nodes(g, *grid);
    int group = 0;
    rc = group_of(b, rp, &group);
    if (rc) return rc;
    int idx = -1;
    for (int i = 0; i < (int)b->h_inst.size(); ++i)
        if (!b->h_inst[i].live) {
            idx = i;
            break;
        }
    if (idx < 0) {
        if ((int)b->h_inst.size() >= b->max_inst) return bfail(SFG_ERR_BUDGET, "all %d instance slots in use", b->max_inst);
        idx = (int)b->h_inst.size();
        b->h_inst.push_back(BatchInst{});
        b->inst_offset.push_back(0);
        b->inst_bytes.push_back(0);
        b->inst_group.push_back(0);
        b->inst_pub.push_back(sfg_grid_desc{});
        b->inst_off.push_back({0, 0, 0});
        b->inst_law.push_back(LawView{});
    }
    const size_t per = align256(sizeof(double) * 5 * (size_t)g.vs);
    const int bufs = b->num.time_recipe == T_RK4 ? 4 : 3;
    const size_t slab_bytes = instance_slab_bytes(b, *grid, g);
    size_t soff = 0;
    rc = slab_alloc(b, slab_bytes, &soff);
    if (rc) return rc;
    const size_t aos_bytes = sizeof(double) * 5 * (size_t)nodes;
    if (aos_bytes > b->staging_cap) {
        if (b->staging) cudaFree(b->staging);
        b->staging = nullptr;
        b->staging_cap = 0;
        if (cudaMalloc((void**)&b->staging, aos_bytes) != cudaSuccess) {
            slab_free(b, soff, slab_bytes);
            return bfail(SFG_ERR_NOMEM, "staging allocation failed");
        }
        b->staging_cap = aos_bytes;
    }
    BatchInst r{};
    r.g = g;
    r.qn = reinterpret_cast<double*>(b->slab + soff);
    r.qa = reinterpret_cast<double*>(b->slab + soff + per);
    r.qb = reinterpret_cast<double*>(b->slab + soff + 2 * per);
    r.k = bufs == 4 ? reinterpret_cast<double*>(b->slab + soff + 3 * per) : nullptr;
    r.law = nullptr;
    if (pts > 0) {  // the law view and its codes after the state buffers
        char* lbase = b->slab + soff + per * bufs;
        unsigned char* dcodes = reinterpret_cast<unsigned char*>(lbase + align256(sizeof(LawView)));
        lv.codes = dcodes;
        BCUDA(cudaMemcpyAsync(dcodes, codes.data(), codes.size(), cudaMemcpyHostToDevice, b->stream));
        BCUDA(cudaMemcpyAsync(lbase, &lv, sizeof lv, cudaMemcpyHostToDevice, b->stream));
        r.law = reinterpret_cast<const LawView*>(lbase);
        if (!b->has_laws) {  // the step graph gets its law launches
            b->has_laws = true;
            if (b->graph) {
                cudaGraphExecDestroy(b->graph);
                b->graph = nullptr;
            }
        }
    }
    std::memset(&r.clock, 0, sizeof r.clock);
    r.clock.t = 0.0;
    r.clock.t_end = t_end;
    r.clock.next_out = kInfB;
    r.clock.max_dt = num.max_dt > 0.0 ? num.max_dt : kInfB;
    r.clock.limit = kInfB;
    r.clock.dt_bits = 0x7FEFFFFFFFFFFFFFull;
    r.clock.dt_ready = 1;  // reduced below, before the grid's first step
    r.clock.max_steps = max_steps > 0 ? max_steps : std::numeric_limits<long long>::max();
    r.clock.active = 0;
    r.flags = 0;
    r.live = 1;
    std::vector<double> dev_layout;
    if (extra) to_device_layout(*grid, g, off, host_nodes_aos, dev_layout);
    BCUDA(cudaMemcpyAsync(b->staging, extra ? dev_layout.data() : host_nodes_aos, aos_bytes, cudaMemcpyHostToDevice,
                          b->stream));
    if (launch_aos_to_soa(b->staging, r.qn, nodes, g.vs, b->stream) != cudaSuccess)
        return bfail(SFG_ERR_CUDA, "upload transpose failed");
    if (extra) {
        // stage kernels write solved nodes only, and stage outputs are read as
        // the next state: every stage buffer holds the ghost value in its extra
        // nodes, as on a single grid
        BCUDA(cudaMemcpyAsync(r.qa, r.qn, per, cudaMemcpyDeviceToDevice, b->stream));
        BCUDA(cudaMemcpyAsync(r.qb, r.qn, per, cudaMemcpyDeviceToDevice, b->stream));
    }
    BCUDA(cudaMemcpyAsync(b->d_inst + idx, &r, sizeof r, cudaMemcpyHostToDevice, b->stream));
    {
        const long long solved = (long long)(g.hi[0] - g.lo[0]) * (g.hi[1] - g.lo[1]);
        const int blocks = (int)std::min<long long>((solved + TILE_THREADS - 1) / TILE_THREADS, 1024);
        batch_initial_cfl_kernel<<<blocks, TILE_THREADS, 0, b->stream>>>(b->d_inst, idx);
        BCUDA(cudaGetLastError());
    }
    b->h_inst[idx] = r;
    b->inst_offset[idx] = soff;
    b->inst_bytes[idx] = slab_bytes;
    b->inst_group[idx] = group;
    b->inst_pub[idx] = *grid;
    b->inst_off[idx] = {off[0], off[1], off[2]};
    b->inst_law[idx] = lv;
    rc = publish_items(b);  // synchronises the stream
    if (rc) return rc;
    *slot = idx;
    return SFG_OK;
}

int sfg_batch_set_write_interval(sfg_batch b, int slot, double write_interval) {
    if (!b || slot < 0 || slot >= (int)b->h_inst.size() || !b->h_inst[slot].live)
        return bfail(SFG_ERR_NOT_FOUND, "no live instance in slot %d", slot);
    if (!std::isfinite(write_interval)) return bfail(SFG_ERR_ARG, "write interval must be finite");
    BatchInst r;
    BCUDA(cudaMemcpyAsync(&r, b->d_inst + slot, sizeof r, cudaMemcpyDeviceToHost, b->stream));
    BCUDA(cudaStreamSynchronize(b->stream));
    const double wi = write_interval > 0.0 ? write_interval : 0.0;
    r.clock.write_interval = wi;
    r.clock.next_out = wi > 0.0 ? r.clock.t + wi : kInfB;
    BCUDA(cudaMemcpyAsync(&b->d_inst[slot].clock, &r.clock, sizeof r.clock, cudaMemcpyHostToDevice, b->stream));
    BCUDA(cudaStreamSynchronize(b->stream));
    b->h_inst[slot].clock.write_interval = r.clock.write_interval;
    b->h_inst[slot].clock.next_out = r.clock.next_out;
    return SFG_OK;
}

int sfg_batch_remove(sfg_batch b, int slot) {
    if (!b || slot < 0 || slot >= (int)b->h_inst.size() || !b->h_inst[slot].live)
        return bfail(SFG_ERR_NOT_FOUND, "no live instance in slot %d", slot);
    BCUDA(cudaStreamSynchronize(b->stream));
    b->h_inst[slot].live = 0;
    const int zero = 0;
    BCUDA(cudaMemcpyAsync(&b->d_inst[slot].live, &zero, sizeof zero, cudaMemcpyHostToDevice, b->stream));
    BCUDA(cudaStreamSynchronize(b->stream));  // ordered on the batch's (non-blocking) stream
    slab_free(b, b->inst_offset[slot], b->inst_bytes[slot]);
    return publish_items(b);
}

int sfg_batch_step(sfg_batch b, int steps, int graph_steps, int* active) {
    sfg::NvtxRange nvtx_("sfg_batch_step");
    if (!b) return bfail(SFG_ERR_ARG, "null batch");
    if (graph_steps <= 0) graph_steps = 16;
    if (!b->graph || b->graph_steps != graph_steps) {
        if (b->graph) cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
        cudaGraph_t g;
        BCUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        int crc = SFG_OK;
        for (int i = 0; i < graph_steps && !crc; ++i) crc = enqueue_batch_step(b);
        cudaError_t e = cudaStreamEndCapture(b->stream, &g);
        if (crc) return crc;
        if (e != cudaSuccess) return bfail(SFG_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
        e = cudaGraphInstantiate(&b->graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return bfail(SFG_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
        b->graph_steps = graph_steps;
    }
    int done = 0, last_active = -1;
    while (done < steps) {
        if (steps - done >= graph_steps) {
            BCUDA(cudaGraphLaunch(b->graph, b->stream));
            done += graph_steps;
        } else {
            int rc = enqueue_batch_step(b);
            if (rc) return rc;
            done += 1;
        }
        BCUDA(cudaMemcpyAsync(b->h_ctl, b->d_ctl, sizeof(BatchCtl), cudaMemcpyDeviceToHost, b->stream));
        BCUDA(cudaStreamSynchronize(b->stream));
        const int now = b->h_ctl->stepped;
        if (last_active < 0 || now < last_active) {
            // some instances finished: drop their tiles from the work list
            std::vector<BatchInst> tmp(b->h_inst.size());
            if (!tmp.empty()) {
                BCUDA(cudaMemcpy(tmp.data(), b->d_inst, tmp.size() * sizeof(BatchInst), cudaMemcpyDeviceToHost));
                bool changed = false;
                for (size_t i = 0; i < tmp.size(); ++i)
                    if (b->h_inst[i].live && tmp[i].done && !b->h_inst[i].done) {
                        b->h_inst[i].done = 1;
                        changed = true;
                    }
                if (changed) {
                    int rc = publish_items(b);
                    if (rc) return rc;
                }
            }
        }
        last_active = now;
        if (now == 0) break;  // every live instance has finished
    }
    b->batch_steps += done;
    if (active) *active = b->h_ctl->stepped;
    return SFG_OK;
}

int sfg_batch_status(sfg_batch b, int slot, double* time, int64_t* steps, int* running, uint32_t* flags) {
    if (!b || slot < 0 || slot >= (int)b->h_inst.size() || !b->h_inst[slot].live)
        return bfail(SFG_ERR_NOT_FOUND, "no live instance in slot %d", slot);
    BatchInst r;
    BCUDA(cudaMemcpyAsync(&r, b->d_inst + slot, sizeof r, cudaMemcpyDeviceToHost, b->stream));
    BCUDA(cudaStreamSynchronize(b->stream));
    if (time) *time = r.clock.t;
    if (steps) *steps = r.clock.steps;
    if (flags) *flags = r.flags;
    if (running) {
        const double eps = 2.220446049250313e-16;
        double scale = std::max({std::fabs(r.clock.t), std::fabs(r.clock.t_end), 1.0});
        const bool finished = !(r.clock.t_end - r.clock.t > 64.0 * eps * scale) || r.clock.steps >= r.clock.max_steps;
        *running = (finished || r.flags) ? 0 : 1;
    }
    return SFG_OK;
}

int sfg_batch_download(sfg_batch b, int slot, double* host_nodes_aos) {
    sfg::NvtxRange nvtx_("sfg_batch_download");
    if (!b || !host_nodes_aos) return bfail(SFG_ERR_ARG, "null argument");
    if (slot < 0 || slot >= (int)b->h_inst.size() || !b->h_inst[slot].live)
        return bfail(SFG_ERR_NOT_FOUND, "no live instance in slot %d", slot);
    const BatchInst& r = b->h_inst[slot];
    const long long nodes = (long long)r.g.n[0] * r.g.n[1] * r.g.n[2];
    const size_t bytes = sizeof(double) * 5 * (size_t)nodes;
    if (launch_soa_to_aos(r.g, r.qn, b->staging, b->stream) != cudaSuccess)
        return bfail(SFG_ERR_CUDA, "download transpose failed");
    const sfg_grid_desc& pub = b->inst_pub[slot];
    if (!has_extra_nodes(r.g, pub)) {
        BCUDA(cudaMemcpyAsync(host_nodes_aos, b->staging, bytes, cudaMemcpyDeviceToHost, b->stream));
        BCUDA(cudaStreamSynchronize(b->stream));
        return SFG_OK;
    }
    std::vector<double> dev((size_t)nodes * 5);
    BCUDA(cudaMemcpyAsync(dev.data(), b->staging, bytes, cudaMemcpyDeviceToHost, b->stream));
    BCUDA(cudaStreamSynchronize(b->stream));
    to_caller_layout(pub, r.g, b->inst_off[slot].data(), dev.data(), host_nodes_aos);
    return SFG_OK;
}

int sfg_batch_set_variant(sfg_batch b, int variant) {
    if (!b) return bfail(SFG_ERR_ARG, "null batch");
    if (variant != 1 && variant != 2) return bfail(SFG_ERR_ARG, "batched tile variant must be 1 or 2");
    if (variant == b->variant) return SFG_OK;
    b->variant = variant;
    int rc = bind_kernels(b);
    if (rc) return rc;
    return publish_items(b);
}

int sfg_batch_snapshot(sfg_batch b, int count, int* running, double* time, int64_t* steps, uint32_t* flags) {
    if (!b || count < 0) return bfail(SFG_ERR_ARG, "bad argument");
    const int n = std::min<int>(count, (int)b->h_inst.size());
    if (n == 0) return SFG_OK;
    std::vector<BatchInst> tmp(n);
    BCUDA(cudaMemcpyAsync(tmp.data(), b->d_inst, n * sizeof(BatchInst), cudaMemcpyDeviceToHost, b->stream));
    BCUDA(cudaStreamSynchronize(b->stream));
    for (int i = 0; i < n; ++i) {
        const bool live = b->h_inst[i].live != 0;
        const Clock& c = tmp[i].clock;
        const double eps = 2.220446049250313e-16;
        const double scale = std::max({std::fabs(c.t), std::fabs(c.t_end), 1.0});
        const bool finished = !(c.t_end - c.t > 64.0 * eps * scale) || c.steps >= c.max_steps;
        if (running) running[i] = live ? ((finished || tmp[i].flags) ? 0 : 1) : -1;
        if (time) time[i] = c.t;
        if (steps) steps[i] = c.steps;
        if (flags) flags[i] = tmp[i].flags;
    }
    return SFG_OK;
}

int sfg_batch_info(sfg_batch b, size_t* used_bytes, size_t* budget_bytes, int* live, int* items) {
    if (!b) return bfail(SFG_ERR_ARG, "null batch");
    if (used_bytes) *used_bytes = b->used;
    if (budget_bytes) *budget_bytes = b->budget;
    if (live) {
        int n = 0;
        for (const auto& r : b->h_inst) n += r.live;
        *live = n;
    }
    if (items) *items = (int)b->h_items.size();
    return SFG_OK;
}

}  // extern "C"
