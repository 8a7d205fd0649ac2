// sfg_cluster1d.cu -- whole runs of small 1-D grids in one launch: a single
// thread-block cluster of CL_CTAS CTAs steps the grid from sfg_advance's
// start to its end time (or step limit) without returning to the host, with
// the state held in the cluster's distributed shared memory.
//
// A 1000-cell tube costs ~30 us per step on the graph path, almost all of it
// launch latency (dt, finalize, three stage launches, commit per step, each a
// few microseconds of work).  Here:
//   * CTA r owns the nodes [r per, (r + 1) per) of every stage buffer (qn,
//     qa, qb and the RK4 accumulator) in its shared memory for the whole run;
//     HBM is touched only to load the state at the start and store it at
//     the end;
//   * a face stencil reads its nodes from the owning CTA's shared memory
//     (its own, or a neighbour's through distributed shared memory);
//   * one lane computes one face; the upper face of a node comes from the
//     next lane by a warp shuffle, so a warp of 32 faces finishes 31 nodes
//     (the face at a warp boundary is computed by both warps);
//   * one hardware cluster barrier (barrier.cluster: release / acquire at
//     cluster scope) closes each stage; the last stage of a step also
//     publishes each CTA's CFL maximum and status bits into CTA 0's shared
//     memory, so every CTA reads the same dt and stop decision after that
//     barrier (slots double-buffered by step parity: a slot is rewritten two
//     steps later, after a barrier that every reader has passed).
// The clock arithmetic is that of finalize_dt_kernel and commit_kernel
// (Time::Driver, SF_time.cpp:42-93), replayed in every thread; the face flux
// and the stage update are the functions the other kernels use (face_flux,
// finish_node).
//
// FP64 (the plain path), transmissive / periodic / frozen ends, all fluxes
// but Lax-Wendroff, up to CL_MAX_NODES nodes.
#include <cooperative_groups.h>

#include "sfg_internal.h"
#include "sfg_math.cuh"
#include "sfg_stage.cuh"

namespace cg = cooperative_groups;

namespace sfg {

constexpr int CL_CTAS = 8;
constexpr int CL_THREADS = 256;
constexpr int CL_WARPS = CL_THREADS / 32;
constexpr int CL_MAX_NODES = 8192;  // per CTA 1024 nodes: 4 buffers x 5 x 1024 doubles = 160 KB
constexpr int CL_NODES_PER_PASS = CL_WARPS * 31;

namespace {

// Stage buffers (0 = qn, 1 = qa, 2 = qb, 3 = RK4 accumulator) read and
// written by each stage: the same roles stage_view gives the global arrays.
// Euler alternates qn / qa by step parity instead of copying back.
__device__ __forceinline__ void stage_buffers(int time_id, int stage, int parity, int& in, int& out) {
    if (time_id == T_EULER) {
        in = parity;
        out = 1 - parity;
    } else if (time_id == T_SSPRK3) {
        in = stage;
        out = stage == 2 ? 0 : stage + 1;
    } else {
        in = stage == 3 ? 1 : stage;
        out = stage == 0 ? 1 : stage == 1 ? 2 : stage == 2 ? 1 : 0;
    }
}

__host__ __device__ __forceinline__ int buffer_count(int time_id) {
    return time_id == T_EULER ? 2 : time_id == T_SSPRK3 ? 3 : 4;
}

}  // namespace

template <int SCHEME, int FLUX>
__global__ void __cluster_dims__(CL_CTAS, 1, 1) __launch_bounds__(CL_THREADS)
    cluster1d_kernel(GridView g, ClusterRun run) {
    constexpr int NST = SchemeInfo<SCHEME>::NST;
    extern __shared__ double cl_smem[];                 // [buffer][5][per]
    __shared__ double slots[2][CL_CTAS];                // CFL maxima (in CTA 0), by step parity
    __shared__ unsigned fslots[2][CL_CTAS];             // status bits (in CTA 0)
    __shared__ double warp_max[CL_WARPS];
    __shared__ unsigned warp_flags[CL_WARPS];
    cg::cluster_group cluster = cg::this_cluster();
    const int rank = (int)cluster.block_rank();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int n = g.n[0];
    const int per = (n + CL_CTAS - 1) / CL_CTAS;
    const int c0 = rank * per, c1 = min(n, c0 + per);        // owned nodes
    const int s0 = max(c0, g.lo[0]), s1 = min(c1, g.hi[0]);  // owned solved nodes (s1 <= s0: none)
    const int time_id = run.sv[0].time_id;
    const int nbuf = buffer_count(time_id);
    const int bstride = 5 * per;                              // doubles per buffer
    const long long vs = g.vs;
    GridView gl = g;                                          // node index = local index, stride per
    gl.vs = per;

    // load the owned chunk of qn into every buffer (unsolved nodes -- frozen
    // ghost values -- stay as loaded in all of them)
    for (int i = c0 + threadIdx.x; i < c1; i += CL_THREADS) {
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            const double x = __ldcg(run.sv[0].qs + v * vs + i);
            for (int b = 0; b < nbuf; ++b) cl_smem[b * bstride + v * per + (i - c0)] = x;
        }
    }

    // the CTA's CFL maximum and status bits -> slot `par` of CTA 0 (every
    // thread calls; visible to the cluster after the next cluster barrier)
    auto publish = [&](double sr, unsigned fl, int par) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sr = fmax(sr, __shfl_xor_sync(0xffffffffu, sr, o));
        fl = __reduce_or_sync(0xffffffffu, fl);
        if (lane == 0) {
            warp_max[warp] = sr;
            warp_flags[warp] = fl;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double m = warp_max[0];
            unsigned f = warp_flags[0];
            for (int w = 1; w < CL_WARPS; ++w) {
                m = fmax(m, warp_max[w]);
                f |= warp_flags[w];
            }
            cluster.map_shared_rank(&slots[par][0], 0)[rank] = m;
            cluster.map_shared_rank(&fslots[par][0], 0)[rank] = f;
            if (f) atomicOr(run.flags, f);
        }
    };
    // after the barrier: the cluster's maximum and status bits (every thread)
    auto gather = [&](int par, double& m, unsigned& f) {
        double x = 0.0;
        unsigned b = 0;
        if (lane < CL_CTAS) {
            x = cluster.map_shared_rank(&slots[par][0], 0)[lane];
            b = cluster.map_shared_rank(&fslots[par][0], 0)[lane];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x = fmax(x, __shfl_xor_sync(0xffffffffu, x, o));
        m = x;
        f = __reduce_or_sync(0xffffffffu, b);
    };

    // the CFL maximum of the state the run starts from (slot parity 1; step
    // `it` publishes into parity it & 1)
    {
        double sr = 0.0;
        unsigned fl = 0;
        __syncthreads();
        for (int i = s0 + threadIdx.x; i < s1; i += CL_THREADS) {
            double q[5];
#pragma unroll
            for (int v = 0; v < 5; ++v) q[v] = cl_smem[v * per + (i - c0)];
            const double r = cfl_rate(g, q);
            if (!(r > 0.0) || !isfinite(r)) fl |= FLAG_NONFINITE;  // as dt_kernel
            sr = fmax(sr, r);
        }
        publish(sr, fl, 1);
    }
    cluster.sync();  // the loaded chunks and the first slots are visible cluster-wide
    double sr_max;
    unsigned bad;
    gather(1, sr_max, bad);
    if (bad) sr_max = 0.0;  // an invalid state: no step

    Clock c = *run.clock;
    const long long first = c.steps;
    const double eps = 2.220446049250313e-16;
    bool more = false;  // stopped by the per-launch step bound, not by the run's end
    int parity = 0;     // Euler: buffer holding the current state
    unsigned cores = 0, cut = 0;
    const int passes = s1 > s0 ? (s1 - s0 + CL_NODES_PER_PASS - 1) / CL_NODES_PER_PASS : 0;
    for (int it = 0;; ++it) {
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

        double sr = 0.0;
        unsigned flags = 0;
        for (int s = 0; s < run.stages; ++s) {
            int bin, bout;
            stage_buffers(time_id, s, parity, bin, bout);
            StageView sv = run.sv[s];
            sv.qout = cl_smem + bout * bstride;
            sv.q0 = cl_smem;                  // qn
            sv.k = cl_smem + 3 * bstride;     // RK4 only
            sv.mode = MODE_FINAL | (s == run.stages - 1 ? MODE_CFL : 0);
            const double* in_local = cl_smem + bin * bstride;
            for (int p = 0; p < passes; ++p) {
                const int f = s0 + p * CL_NODES_PER_PASS + warp * 31 + lane;  // face f: lower face of node f
                double Fa[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
                if (f <= s1) {
                    double st[NST][5];
#pragma unroll
                    for (int k = 0; k < NST; ++k) {
                        const int j = map_index(f - NST / 2 + k, n, g.bc_lo[0], g.bc_hi[0]);
                        const int owner = j / per;
                        const double* src =
                            owner == rank ? in_local : cluster.map_shared_rank(in_local, owner);
#pragma unroll
                        for (int v = 0; v < 5; ++v) st[k][v] = src[v * per + (j - owner * per)];
                    }
                    double F[5];
                    face_flux<0, SCHEME, FLUX, double>(st, g.gamma, F, flags, cut, 0.0);
#pragma unroll
                    for (int v = 0; v < 5; ++v) Fa[v] = F[v] * g.area[0];
                    if (SCHEME == TENO5 && (lane < 31 || f == s1)) cores += 10;
                }
                double div[5];
#pragma unroll
                for (int v = 0; v < 5; ++v) div[v] = __shfl_down_sync(0xffffffffu, Fa[v], 1) - Fa[v];
                if (lane < 31 && f < s1) {
                    const int li = f - c0;
                    double qn[5];
#pragma unroll
                    for (int v = 0; v < 5; ++v) qn[v] = in_local[v * per + li];
                    finish_node(gl, sv, dt, li, qn, div, flags, sr);
                }
            }
            if (s == run.stages - 1) publish(sr, flags, it & 1);
            cluster.sync();  // the stage's output is visible cluster-wide
        }
        if (time_id == T_EULER) parity ^= 1;
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
        gather(it & 1, sr_max, bad);
        if (bad) break;  // an invalid state stops the run (the same bits in every CTA)
    }
    // the owned solved nodes of the current state back to qn
    const double* cur = cl_smem + (time_id == T_EULER ? parity : 0) * bstride;
    double* qn_out = const_cast<double*>(run.sv[0].qs);
    for (int i = s0 + threadIdx.x; i < s1; i += CL_THREADS) {
#pragma unroll
        for (int v = 0; v < 5; ++v) qn_out[v * vs + i] = cur[v * per + (i - c0)];
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
    cluster.sync();  // no CTA leaves while another may still read its shared memory
}

template <int SCHEME, int FLUX>
static cudaError_t launch_cluster(const GridView& g, const ClusterRun& run, size_t smem, cudaStream_t st) {
    auto kern = cluster1d_kernel<SCHEME, FLUX>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<CL_CTAS, CL_THREADS, smem, st>>>(g, run);
    return cudaGetLastError();
}

template <int SCHEME>
static cudaError_t launch_cluster_f(int flux, const GridView& g, const ClusterRun& run, size_t smem,
                                    cudaStream_t st) {
    switch (flux) {
    case RUSANOV: return launch_cluster<SCHEME, RUSANOV>(g, run, smem, st);
    case ROE: return launch_cluster<SCHEME, ROE>(g, run, smem, st);
    case STEGER: return launch_cluster<SCHEME, STEGER>(g, run, smem, st);
    case LAXF: return launch_cluster<SCHEME, LAXF>(g, run, smem, st);
    }
    return cudaErrorInvalidValue;
}

// Whether a 1-D grid can run in the cluster kernel.
bool cluster1d_eligible(const GridView& g, int flux, int prec64) {
    return g.dim == 1 && prec64 && flux != LAXW && !g.curv && g.hi[0] - g.lo[0] >= CL_CTAS &&
           g.n[0] <= CL_MAX_NODES;
}

cudaError_t launch_cluster1d(int scheme, int flux, const GridView& g, const ClusterRun& run, cudaStream_t st) {
    const int per = (g.n[0] + CL_CTAS - 1) / CL_CTAS;
    const size_t smem = sizeof(double) * 5 * (size_t)per * buffer_count(run.sv[0].time_id);
    switch (scheme) {
    case WENO5: return launch_cluster_f<WENO5>(flux, g, run, smem, st);
    case TENO5: return launch_cluster_f<TENO5>(flux, g, run, smem, st);
    case WENO3: return launch_cluster_f<WENO3>(flux, g, run, smem, st);
    case WENO7: return launch_cluster_f<WENO7>(flux, g, run, smem, st);
    }
    return cudaErrorInvalidValue;
}

}  // namespace sfg
