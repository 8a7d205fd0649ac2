// sfg_cluster1d.cu -- whole runs of small 1-D grids in one launch: a single
// thread-block cluster of CL_CTAS CTAs steps the grid from sfg_advance's
// start to its end time (or step limit) without returning to the host.
//
// A 1000-cell tube costs ~30 us per step on the graph path, almost all of it
// launch latency (dt, finalize, three stage launches, commit per step, each a
// few microseconds of work).  Here the launches become cluster barriers
// (barrier.cluster, a hardware barrier with release / acquire ordering at
// cluster scope): per stage, every CTA computes the face fluxes of its node
// chunk into a face array, the cluster synchronises, every CTA updates its
// nodes, and the cluster synchronises again.  The CFL maximum of each CTA
// goes into CTA 0's shared memory through distributed shared memory; every
// CTA reads the same slots back, so all CTAs hold the same dt and take the
// same loop decisions.  The clock arithmetic is that of finalize_dt_kernel
// and commit_kernel (Time::Driver, SF_time.cpp:42-93), replayed in every CTA.
//
// FP64 (the plain path), transmissive / periodic / frozen ends, all fluxes
// but Lax-Wendroff; the face fluxes and the stage update are the functions
// the other kernels use (face_flux, finish_node).
#include <cooperative_groups.h>

#include "sfg_internal.h"
#include "sfg_math.cuh"
#include "sfg_stage.cuh"

namespace cg = cooperative_groups;

namespace sfg {

constexpr int CL_CTAS = 8;
constexpr int CL_THREADS = 256;
constexpr int CL_MAX_NODES = CL_CTAS * CL_THREADS * 4;  // up to 4 nodes per thread

namespace {

// The largest value over the cluster: each CTA's maximum goes to slot r of
// CTA 0's shared array, then every CTA reads all slots.  Every thread of
// every CTA calls it.
__device__ double cluster_max(double x, double* slots, cg::cluster_group& cluster) {
    __shared__ double warp_max[CL_THREADS / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x = fmax(x, __shfl_xor_sync(0xffffffffu, x, o));
    if ((threadIdx.x & 31) == 0) warp_max[threadIdx.x >> 5] = x;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = warp_max[0];
        for (int w = 1; w < CL_THREADS / 32; ++w) m = fmax(m, warp_max[w]);
        double* dst = cluster.map_shared_rank(slots, 0);
        dst[cluster.block_rank()] = m;
    }
    cluster.sync();
    const double* src = cluster.map_shared_rank(slots, 0);
    double m = src[0];
    for (int r = 1; r < CL_CTAS; ++r) m = fmax(m, src[r]);
    cluster.sync();  // slots are read before anyone writes them again
    return m;
}

}  // namespace

template <int SCHEME, int FLUX>
__global__ void __cluster_dims__(CL_CTAS, 1, 1) __launch_bounds__(CL_THREADS)
    cluster1d_kernel(GridView g, ClusterRun run) {
    constexpr int NST = SchemeInfo<SCHEME>::NST;
    __shared__ double slots[CL_CTAS];
    cg::cluster_group cluster = cg::this_cluster();
    const int rank = (int)cluster.block_rank();
    const long long vs = g.vs;
    // node chunk of this CTA over the solved range [lo, hi) (empty for the
    // trailing CTAs of a short grid: n1 < n0); faces i in [lo, hi] (face i is
    // the lower face of node i, face hi the upper face of the last node),
    // split the same way, the extra face hi going to the CTA that holds the
    // last node.  On a periodic axis face n is face 0 and is not computed twice.
    const int lo = g.lo[0], hi = g.hi[0], count = hi - lo;
    const int per = (count + CL_CTAS - 1) / CL_CTAS;
    const int n0 = lo + rank * per, n1 = min(hi, n0 + per);
    const bool periodic = g.bc_lo[0] == BC_PERIODIC;
    const int f0 = n0, f1 = (n0 < hi && n1 == hi && !periodic) ? hi + 1 : n1;
    unsigned flags = 0, cut = 0, cores = 0;

    // the CFL maximum of the state the run starts from
    double sr = 0.0;
    for (int i = n0 + threadIdx.x; i < n1; i += CL_THREADS) {
        const double* qs = run.sv[0].qs;
        const double q[5] = {__ldcg(qs + i), __ldcg(qs + vs + i), __ldcg(qs + 2 * vs + i), __ldcg(qs + 3 * vs + i),
                             __ldcg(qs + 4 * vs + i)};
        const double r = cfl_rate(g, q);
        if (!(r > 0.0) || !isfinite(r)) flags |= FLAG_NONFINITE;  // as dt_kernel
        sr = fmax(sr, r);
    }
    if (flags) atomicOr(run.flags, flags);
    flags = 0;
    double sr_max = cluster_max(sr, slots, cluster);
    if (*(volatile unsigned*)run.flags) sr_max = 0.0;  // an invalid state: no step (every CTA agrees)
    Clock c = *run.clock;
    const long long first = c.steps;
    const double eps = 2.220446049250313e-16;
    bool more = false;   // stopped by the per-launch step bound, not by the run's end
    for (;;) {
        // finalize_dt_kernel
        const double remaining = c.t_end - c.t;
        double scale = fmax(fabs(c.t), fabs(c.t_end));
        scale = scale < 1.0 ? 1.0 : scale;
        if (!(remaining > 64.0 * eps * scale) || c.steps >= c.max_steps || !(sr_max > 0.0)) break;
        if (c.steps - first >= run.launch_steps) {
            more = true;
            break;
        }
        double limit = remaining;
        if (c.write_interval > 0.0 && c.next_out - c.t < limit) limit = c.next_out - c.t;
        if (c.limit < limit) limit = c.limit;
        double dt = __ddiv_rn(g.cfl, sr_max);
        if (c.max_dt < dt) dt = c.max_dt;
        if (limit < dt) dt = limit;
        // the stages
        sr = 0.0;
        for (int s = 0; s < run.stages; ++s) {
            const StageView& sv = run.sv[s];
            for (int i = f0 + threadIdx.x; i < f1; i += CL_THREADS) {
                double st[NST][5];
#pragma unroll
                for (int k = 0; k < NST; ++k) {
                    const int node = map_index(i - NST / 2 + k, g.n[0], g.bc_lo[0], g.bc_hi[0]);
#pragma unroll
                    for (int v = 0; v < 5; ++v) st[k][v] = __ldcg(sv.qs + v * vs + node);
                }
                double F[5];
                face_flux<0, SCHEME, FLUX, double>(st, g.gamma, F, flags, cut, 0.0);
                const int face = i < g.n[0] ? i : i - g.n[0];  // periodic: face n is face 0
#pragma unroll
                for (int v = 0; v < 5; ++v) run.faces[v * vs + face] = F[v] * g.area[0];
                if (SCHEME == TENO5) cores += 10;
            }
            cluster.sync();
            StageView svs = sv;
            svs.mode = MODE_FINAL | (s == run.stages - 1 ? MODE_CFL : 0);
            for (int i = n0 + threadIdx.x; i < n1; i += CL_THREADS) {
                const int up = i + 1 < g.n[0] ? i + 1 : i + 1 - g.n[0];
                double div[5], qn[5];
#pragma unroll
                for (int v = 0; v < 5; ++v) {
                    div[v] = __ldcg(run.faces + v * vs + up) - __ldcg(run.faces + v * vs + i);
                    qn[v] = __ldcg(sv.qs + v * vs + i);
                }
                finish_node(g, svs, dt, i, qn, div, flags, sr);
            }
            if (flags) atomicOr(run.flags, flags);
            flags = 0;
            cluster.sync();
        }
        // commit_kernel
        if (rank == 0 && threadIdx.x == 0 && run.dt_log && c.steps - c.log_base < run.dt_cap &&
            c.steps >= c.log_base)
            run.dt_log[c.steps - c.log_base] = dt;
        c.t += dt;
        c.steps += 1;
        double sc = fabs(c.t);
        sc = sc < 1.0 ? 1.0 : sc;
        if (c.write_interval > 0.0 && c.t >= c.next_out - 1.0e-11 * sc) c.next_out += c.write_interval;
        c.limit = __longlong_as_double(0x7FF0000000000000ll);
        c.dt = dt;
        sr_max = cluster_max(sr, slots, cluster);
        // a failed state stops the run (every CTA sees the same word after
        // the barriers of cluster_max)
        if (*(volatile unsigned*)run.flags) break;
    }
    if (rank == 0 && threadIdx.x == 0) {
        c.active = more ? 1 : 0;
        c.dt_ready = 0;
        c.dt_bits = 0x7FEFFFFFFFFFFFFFull;
        *run.clock = c;
    }
    if (run.sv[0].counters && (cores | cut)) {
        atomicAdd(run.sv[0].counters + 0, (unsigned long long)cores);
        atomicAdd(run.sv[0].counters + 1, (unsigned long long)cut);
    }
}

template <int SCHEME, int FLUX>
static cudaError_t launch_cluster(const GridView& g, const ClusterRun& run, cudaStream_t st) {
    cluster1d_kernel<SCHEME, FLUX><<<CL_CTAS, CL_THREADS, 0, st>>>(g, run);
    return cudaGetLastError();
}

template <int SCHEME>
static cudaError_t launch_cluster_f(int flux, const GridView& g, const ClusterRun& run, cudaStream_t st) {
    switch (flux) {
    case RUSANOV: return launch_cluster<SCHEME, RUSANOV>(g, run, st);
    case ROE: return launch_cluster<SCHEME, ROE>(g, run, st);
    case STEGER: return launch_cluster<SCHEME, STEGER>(g, run, st);
    case LAXF: return launch_cluster<SCHEME, LAXF>(g, run, st);
    }
    return cudaErrorInvalidValue;
}

// Whether a 1-D grid can run in the cluster kernel.
bool cluster1d_eligible(const GridView& g, int flux, int prec64) {
    return g.dim == 1 && prec64 && flux != LAXW && !g.curv && g.hi[0] - g.lo[0] >= CL_CTAS &&
           g.n[0] <= CL_MAX_NODES;
}

cudaError_t launch_cluster1d(int scheme, int flux, const GridView& g, const ClusterRun& run, cudaStream_t st) {
    switch (scheme) {
    case WENO5: return launch_cluster_f<WENO5>(flux, g, run, st);
    case TENO5: return launch_cluster_f<TENO5>(flux, g, run, st);
    case WENO3: return launch_cluster_f<WENO3>(flux, g, run, st);
    case WENO7: return launch_cluster_f<WENO7>(flux, g, run, st);
    }
    return cudaErrorInvalidValue;
}

}  // namespace sfg
