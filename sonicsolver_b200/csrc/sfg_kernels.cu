// sfg_kernels.cu -- sm_100a kernels of the explicit Euler path.
//
// State layout in HBM: structure of arrays, q[v * vs + (k * ny + j) * nx + i]
// over the nodes only (no ghost storage).  Ghost and boundary-node values are
// produced by index mapping when a stencil is read:
//   transmissive end: any index at or beyond the boundary node reads its inner
//     neighbour (zeroGradient: boundary node <- inner node, ghosts <- boundary
//     node; reconstruction/linear/SF_zeroGradient.cpp:88-105);
//   periodic end: indices wrap.
// This is the in-device replacement of the per-stage ghost fill and MPI halo
// exchange (SF_conservativeRHS.cpp:75-104).
//
// One stage on a D-dimensional grid is D sweep launches.  Sweep d computes
// the face fluxes along axis d once per face, differences them into the node
// residual (held in registers, accumulated through a FP64 residual array
// across axes), and the last sweep applies the stage combination.
//   x sweeps: one warp per 31 consecutive nodes of a row, one lane per face,
//     neighbour face by warp shuffle (coalesced loads along x);
//   y / z sweeps: one thread per node column segment, marching along the axis
//     with the stencil in a register sliding window (one node load per face).
#include "sfg_internal.h"
#include "sfg_math.cuh"
#include "sfg_stage.cuh"

#include <cstdio>

namespace sfg {

// ---------------------------------------------------------------------------
// x sweep: blockDim = (32, ROWS); one warp per 31 nodes of one row.
// ---------------------------------------------------------------------------
template <int SCHEME, int FLUX, typename T>
__global__ void __launch_bounds__(128, 5) sweep_x(GridView g, StageView sv) {
    constexpr int NST = SchemeInfo<SCHEME>::NST;
    if (sv.require_active && !sv.clock->active) return;
    const int lane = threadIdx.x;
    const int cnt_y = g.hi[1] - g.lo[1];
    const int cnt_z = g.hi[2] - g.lo[2];
    const int row = blockIdx.y * blockDim.y + threadIdx.y;
    if (row >= cnt_y * cnt_z) return;  // whole warp exits together
    const int j = g.lo[1] + row % cnt_y;
    const int k = g.lo[2] + row / cnt_y;
    const int i0 = g.lo[0] + blockIdx.x * 31;
    const int nodes = min(31, g.hi[0] - i0);
    const int f = i0 + lane;  // face between nodes f-1 and f
    const long long rowbase = ((long long)k * g.n[1] + j) * g.n[0];
    const long long vs = g.vs;
    unsigned flags = 0, cut = 0;
    double sr = 0.0;
    double st[NST][5];
    double F[5] = {0, 0, 0, 0, 0};
    if (lane <= nodes) {
#pragma unroll
        for (int s = 0; s < NST; ++s) {
            const int ii = map_index(f - NST / 2 + s, g.n[0], g.bc_lo[0], g.bc_hi[0]);
#pragma unroll
            for (int v = 0; v < 5; ++v) st[s][v] = __ldg(sv.qs + v * vs + rowbase + ii);
        }
        T Ft[5];
        if constexpr (sizeof(T) == sizeof(float)) {
            // deviations from the stage's reference node (ref_node)
            double qref[5];
            load_ref(g, sv.qs, qref);
            const Ref32 ref = make_ref32(qref, g.gamma);
            float d[NST][5];
#pragma unroll
            for (int s = 0; s < NST; ++s)
#pragma unroll
                for (int v = 0; v < 5; ++v) d[s][v] = float(st[s][v] - qref[v]);
            face_flux_dev32<0, SCHEME, FLUX>(d, ref, float(g.gamma), Ft, flags, cut, sv.counters != nullptr);
        } else {
            face_flux<0, SCHEME, FLUX, T>(st, T(g.gamma), Ft, flags, cut, T(FLUX == LAXW ? sv.clock->dt / g.h[0] : 0.0));
        }
#pragma unroll
        for (int v = 0; v < 5; ++v) F[v] = double(Ft[v]) * g.area[0];
    }
    double div[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) div[v] = __shfl_down_sync(0xffffffffu, F[v], 1) - F[v];
    if (lane < nodes) {
        const long long node = rowbase + f;
        if (sv.mode & MODE_READ_R) {
#pragma unroll
            for (int v = 0; v < 5; ++v) div[v] = sv.r[v * vs + node] + div[v];
        }
        if (sv.mode & MODE_FINAL) {
            double qn[5];
#pragma unroll
            for (int v = 0; v < 5; ++v) qn[v] = st[NST / 2][v];
            finish_node(g, sv, sv.clock->dt, node, qn, div, flags, sr);
        } else {
#pragma unroll
            for (int v = 0; v < 5; ++v) sv.r[v * vs + node] = div[v];
        }
    }
    flush_status(sv, flags, SCHEME == TENO5 ? (lane <= nodes ? 10u : 0u) : 0u, cut);
    if (sv.mode & MODE_CFL) flush_cfl_warp(g, sv.clock, sr);
}

// ---------------------------------------------------------------------------
// y / z sweep: blockDim = (32, SEGS); thread = (x node, segment of SEGLEN
// nodes along AX); blockIdx.z = the remaining axis.
// ---------------------------------------------------------------------------
constexpr int SEGLEN = 16;

// FP32-flux segment: the register window holds FP32 deviations from the
// stage's reference node (ref_node; one FP64 -> FP32 rounding per node), the
// face fluxes are deviations F - F(q_ref) (face_flux_dev32).  Every face of
// the launch shares the reference, so F(q_ref) cancels from the divergence
// exactly and a face on a segment boundary has the same bits in both
// segments.  The FP64 node value for the stage update is re-read (L1 / L2).
template <int AX, int SCHEME, int FLUX>
__device__ __forceinline__ void sweep_yz_f32_segment(const GridView& g, const StageView& sv, int i, int o, int s0,
                                                     unsigned& flags, unsigned& cut, unsigned& cores,
                                                     double& sr_max) {
    constexpr int NST = SchemeInfo<SCHEME>::NST;
    constexpr int OTHER = AX == 1 ? 2 : 1;
    const int s1 = min(s0 + SEGLEN, g.hi[AX]);
    const long long vs = g.vs;
    const long long sy = g.n[0], sz = (long long)g.n[0] * g.n[1];
    const long long sa = AX == 1 ? sy : sz;
    const long long base = i + (long long)o * (OTHER == 1 ? sy : sz);
    const int n = g.n[AX];
    const int bl = g.bc_lo[AX], bh = g.bc_hi[AX];
    const double dt = sv.clock->dt;
    double qref[5];
    load_ref(g, sv.qs, qref);
    const Ref32 ref = make_ref32(qref, g.gamma);
    const float gamma = float(g.gamma);
    float d[NST][5];
#pragma unroll
    for (int s = 0; s < NST; ++s) {
        const int a = map_index(s0 - NST / 2 + s, n, bl, bh);
#pragma unroll
        for (int v = 0; v < 5; ++v) d[s][v] = float(sv.qs[v * vs + base + a * sa] - qref[v]);
    }
    double Fp[5];
    for (int f = s0; f <= s1; ++f) {
        float Ft[5];
        face_flux_dev32<AX, SCHEME, FLUX>(d, ref, gamma, Ft, flags, cut, sv.counters != nullptr);
        if (SCHEME == TENO5) cores += 10;
        double F[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) F[v] = double(Ft[v]) * g.area[AX];
        if (f > s0) {
            const long long node = base + (long long)(f - 1) * sa;
            double div[5];
#pragma unroll
            for (int v = 0; v < 5; ++v) div[v] = F[v] - Fp[v];
            if (sv.mode & MODE_READ_R) {
#pragma unroll
                for (int v = 0; v < 5; ++v) div[v] = sv.r[v * vs + node] + div[v];
            }
            if (sv.mode & MODE_FINAL) {
                double qn[5];
#pragma unroll
                for (int v = 0; v < 5; ++v) qn[v] = sv.qs[v * vs + node];
                finish_node(g, sv, dt, node, qn, div, flags, sr_max);
            } else {
#pragma unroll
                for (int v = 0; v < 5; ++v) sv.r[v * vs + node] = div[v];
            }
        }
#pragma unroll
        for (int v = 0; v < 5; ++v) Fp[v] = F[v];
        if (f < s1) {
#pragma unroll
            for (int s = 0; s < NST - 1; ++s)
#pragma unroll
                for (int v = 0; v < 5; ++v) d[s][v] = d[s + 1][v];
            const int a = map_index(f + 1 - NST / 2 + NST - 1, n, bl, bh);
#pragma unroll
            for (int v = 0; v < 5; ++v) d[NST - 1][v] = float(sv.qs[v * vs + base + a * sa] - qref[v]);
        }
    }
}

template <int AX, int SCHEME, int FLUX, typename T>
__global__ void __launch_bounds__(128, 4) sweep_yz(GridView g, StageView sv) {
    constexpr int NST = SchemeInfo<SCHEME>::NST;
    if (sv.require_active && !sv.clock->active) return;
    constexpr int OTHER = AX == 1 ? 2 : 1;
    const int i = g.lo[0] + blockIdx.x * 32 + threadIdx.x;
    const int o = g.lo[OTHER] + blockIdx.z;
    const int s0 = g.lo[AX] + (blockIdx.y * blockDim.y + threadIdx.y) * SEGLEN;
    const bool live = i < g.hi[0] && s0 < g.hi[AX];
    unsigned flags = 0, cut = 0, cores = 0;
    double sr = 0.0;
    if constexpr (sizeof(T) == sizeof(float)) {
        if (live) sweep_yz_f32_segment<AX, SCHEME, FLUX>(g, sv, i, o, s0, flags, cut, cores, sr);
    } else if (live) {
        const int s1 = min(s0 + SEGLEN, g.hi[AX]);
        const long long vs = g.vs;
        const long long sx = 1, sy = g.n[0], sz = (long long)g.n[0] * g.n[1];
        const long long sa = AX == 1 ? sy : sz;
        const long long base = i * sx + (long long)o * (OTHER == 1 ? sy : sz);
        const int n = g.n[AX];
        const int bl = g.bc_lo[AX], bh = g.bc_hi[AX];
        const double dt = sv.clock->dt;
        double st[NST][5];
#pragma unroll
        for (int s = 0; s < NST; ++s) {
            const int a = map_index(s0 - NST / 2 + s, n, bl, bh);
#pragma unroll
            for (int v = 0; v < 5; ++v) st[s][v] = sv.qs[v * vs + base + a * sa];
        }
        double Fp[5];
        for (int f = s0; f <= s1; ++f) {
            T Ft[5];
            face_flux<AX, SCHEME, FLUX, T>(st, T(g.gamma), Ft, flags, cut,
                                           T(FLUX == LAXW ? sv.clock->dt / g.h[AX] : 0.0));
            if (SCHEME == TENO5) cores += 10;
            double F[5];
#pragma unroll
            for (int v = 0; v < 5; ++v) F[v] = double(Ft[v]) * g.area[AX];
            if (f > s0) {
                const long long node = base + (long long)(f - 1) * sa;
                double div[5];
#pragma unroll
                for (int v = 0; v < 5; ++v) div[v] = F[v] - Fp[v];
                if (sv.mode & MODE_READ_R) {
#pragma unroll
                    for (int v = 0; v < 5; ++v) div[v] = sv.r[v * vs + node] + div[v];
                }
                if (sv.mode & MODE_FINAL) {
                    double qn[5];
#pragma unroll
                    for (int v = 0; v < 5; ++v) qn[v] = st[NST / 2 - 1][v];
                    finish_node(g, sv, dt, node, qn, div, flags, sr);
                } else {
#pragma unroll
                    for (int v = 0; v < 5; ++v) sv.r[v * vs + node] = div[v];
                }
            }
#pragma unroll
            for (int v = 0; v < 5; ++v) Fp[v] = F[v];
            if (f < s1) {
#pragma unroll
                for (int s = 0; s < NST - 1; ++s)
#pragma unroll
                    for (int v = 0; v < 5; ++v) st[s][v] = st[s + 1][v];
                const int a = map_index(f + 1 - NST / 2 + NST - 1, n, bl, bh);
#pragma unroll
                for (int v = 0; v < 5; ++v) st[NST - 1][v] = sv.qs[v * vs + base + a * sa];
            }
        }
    }
    flush_status(sv, flags, cores, cut);
    if (sv.mode & MODE_CFL) flush_cfl_warp(g, sv.clock, sr);
}

// ---------------------------------------------------------------------------
// CFL step (RusanovEOS::deltaT, SF_rusanovEOS.cpp:110-147) with the block /
// grid minimum replacing Runtime::globalMinimum's MPI_Allreduce(MIN).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) dt_kernel(GridView g, const double* __restrict__ q, Clock* clock,
                                                 unsigned* flags, int skip_if_ready) {
    if (skip_if_ready && clock->dt_ready) return;  // the previous step's last stage reduced it
    // Work item = 64 consecutive solved nodes of one x row, taken by one
    // warp (2 nodes a lane, loaded together): the node index needs integer
    // divisions once per item, not once per node.
    const int cx = g.hi[0] - g.lo[0], cy = g.hi[1] - g.lo[1], cz = g.hi[2] - g.lo[2];
    const int chunks = (cx + 63) / 64;
    const long long items = (long long)chunks * cy * cz;
    const int lane = threadIdx.x & 31;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    double best = 0.0;  // largest spectral-radius sum; dt = CFL / best
    unsigned fl = 0;
    for (long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < items; w += nwarps) {
        const long long row = w / chunks;
        const int i0 = g.lo[0] + (int)(w - row * chunks) * 64;
        const int iend = min(g.hi[0], i0 + 64);
        const int j = g.lo[1] + (int)(row % cy), k = g.lo[2] + (int)(row / cy);
        const long long base = ((long long)k * g.n[1] + j) * g.n[0];
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int i = i0 + 32 * u + lane;
            if (i < iend) {
                const long long node = base + i;
                const double qq[5] = {q[node], q[g.vs + node], q[2 * g.vs + node], q[3 * g.vs + node],
                                      q[4 * g.vs + node]};
                const double sr = cfl_rate_node(g, qq, node);
                if (!(sr > 0.0) || !isfinite(sr)) fl |= FLAG_NONFINITE;
                best = fmax(best, sr);
            }
        }
    }
    flush_cfl_block(g, clock, best);
    if (fl) atomicOr(flags, fl);
}

// FlowDtCompute's min(dt, maxDeltaT, limit) with the Time::Driver end / output
// clipping and stop test (SF_time.cpp:56-72).  One thread.  A status word
// with bits set stops the run (the reference exits on an invalid state): the
// failing step is the last one counted, and the rest of a graph is no-ops.
__global__ void finalize_dt_kernel(Clock* c, const unsigned* flags) {
    if (*flags) {
        c->active = 0;
        return;
    }
    const double eps = 2.220446049250313e-16;
    const double remaining = c->t_end - c->t;
    double scale = fmax(fabs(c->t), fabs(c->t_end));
    scale = scale < 1.0 ? 1.0 : scale;
    if (!(remaining > 64.0 * eps * scale) || c->steps >= c->max_steps) {
        c->active = 0;  // dt keeps the last step's size
        return;
    }
    double limit = remaining;
    if (c->write_interval > 0.0 && c->next_out - c->t < limit) limit = c->next_out - c->t;
    if (c->limit < limit) limit = c->limit;
    double dt = __longlong_as_double((long long)c->dt_bits);
    if (c->max_dt < dt) dt = c->max_dt;
    if (limit < dt) dt = limit;
    c->dt = dt;
    c->active = 1;
    c->dt_bits = 0x7FEFFFFFFFFFFFFFull;  // consumed: re-armed for the next minimum
    c->dt_ready = 0;
}

// TimeCommit: t += dt, ++step, output-time bookkeeping.  `cfl_next`: the
// step's last stage reduced the CFL minimum of the new state into dt_bits.
__global__ void commit_kernel(Clock* c, double* dt_log, long long dt_cap, int cfl_next) {
    if (c->active) {
        if (dt_log && c->steps - c->log_base < dt_cap && c->steps >= c->log_base) dt_log[c->steps - c->log_base] = c->dt;
        c->t += c->dt;
        c->steps += 1;
        double sc = fabs(c->t);
        sc = sc < 1.0 ? 1.0 : sc;
        if (c->write_interval > 0.0 && c->t >= c->next_out - 1.0e-11 * sc) c->next_out += c->write_interval;
    }
    c->dt_ready = c->active && cfl_next ? 1 : 0;
    c->limit = __longlong_as_double(0x7FF0000000000000ll);
}

__global__ void set_dt_kernel(Clock* c, double dt) {
    c->dt = dt;
    c->active = 1;
}

__global__ void reset_min_kernel(Clock* c) { c->dt_bits = 0x7FEFFFFFFFFFFFFFull; }

// Stage combination with a residual supplied in sv.r (already Jac-scaled).
__global__ void stage_from_residual_kernel(GridView g, StageView sv) {
    const long long cx = g.hi[0] - g.lo[0], cy = g.hi[1] - g.lo[1], cz = g.hi[2] - g.lo[2];
    const long long total = cx * cy * cz;
    unsigned flags = 0;
    const double dt = sv.clock->dt;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int i = g.lo[0] + (int)(t % cx);
        const int j = g.lo[1] + (int)((t / cx) % cy);
        const int k = g.lo[2] + (int)(t / (cx * cy));
        const long long node = ((long long)k * g.n[1] + j) * g.n[0] + i;
        double out[5];
        for (int v = 0; v < 5; ++v)
            out[v] = stage_value(sv, dt, sv.qs[v * g.vs + node], sv.r[v * g.vs + node], v * g.vs + node);
        for (int v = 0; v < 5; ++v) sv.qout[v * g.vs + node] = out[v];
        if (!(out[0] > 0.0)) flags |= FLAG_DENSITY;
    }
    if (flags) atomicOr(sv.flags, flags);
}

// AoS nodes (host layout) <-> SoA state.  On the way out the unsolved
// transmissive boundary nodes are filled from their inner neighbours (the
// commit ghost fill, SF_flowOperations.cpp:647-652).
__global__ void aos_to_soa_kernel(const double* __restrict__ aos, double* __restrict__ soa, long long nodes,
                                  long long vs) {
    // one warp per 128 consecutive nodes, 4 a lane: SoA stores coalesced per variable
    const int lane = threadIdx.x & 31;
    const long long items = (nodes + 127) / 128, nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < items; w += nwarps) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const long long node = w * 128 + 32 * u + lane;
            if (node < nodes) {
#pragma unroll
                for (int v = 0; v < 5; ++v) soa[v * vs + node] = aos[node * 5 + v];
            }
        }
    }
}

__global__ void soa_to_aos_kernel(GridView g, const double* __restrict__ soa, double* __restrict__ aos) {
    // one warp per 128 nodes of one x row, 4 a lane (index divisions once per
    // row chunk); the row's source after the boundary mapping
    const int lane = threadIdx.x & 31;
    const int chunks = (g.n[0] + 127) / 128;
    const long long items = (long long)chunks * g.n[1] * g.n[2], nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < items; w += nwarps) {
        const long long row = w / chunks;
        const int i0 = (int)(w - row * chunks) * 128;
        int j = (int)(row % g.n[1]), k = (int)(row / g.n[1]);
        const long long dst = ((long long)k * g.n[1] + j) * g.n[0];
        if (g.dim > 1) j = map_index(j, g.n[1], g.bc_lo[1], g.bc_hi[1]);
        if (g.dim > 2) k = map_index(k, g.n[2], g.bc_lo[2], g.bc_hi[2]);
        const long long src = ((long long)k * g.n[1] + j) * g.n[0];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int i = i0 + 32 * u + lane;
            if (i < g.n[0]) {
                const int im = g.dim > 0 ? map_index(i, g.n[0], g.bc_lo[0], g.bc_hi[0]) : i;
#pragma unroll
                for (int v = 0; v < 5; ++v) aos[(dst + i) * 5 + v] = soa[v * g.vs + src + im];
            }
        }
    }
}

// Conserved totals over the nodes (trapezoid-free node sums x cell volume),
// FP64 with a per-block tree and one atomic per block per variable.
__global__ void totals_kernel(GridView g, const double* __restrict__ q, double* __restrict__ out, double vol) {
    const long long nodes = (long long)g.n[0] * g.n[1] * g.n[2];
    double acc[5] = {0, 0, 0, 0, 0};
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nodes;
         t += (long long)gridDim.x * blockDim.x) {
        int c[3] = {(int)(t % g.n[0]), (int)((t / g.n[0]) % g.n[1]), (int)(t / ((long long)g.n[0] * g.n[1]))};
        bool extra = false;  // the frozen-ghost node of a frozen end is not a node of the case
        for (int a = 0; a < g.dim; ++a) {
            extra |= (g.bc_lo[a] == BC_FROZEN && c[a] == 0) || (g.bc_hi[a] == BC_FROZEN && c[a] == g.n[a] - 1);
            c[a] = map_index(c[a], g.n[a], g.bc_lo[a], g.bc_hi[a]);
        }
        if (extra) continue;
        const long long node = ((long long)c[2] * g.n[1] + c[1]) * g.n[0] + c[0];
        const double w = g.curv ? 1.0 / g.node_jac[node] : 1.0;  // node volume J on curvilinear grids
        for (int v = 0; v < 5; ++v) acc[v] += q[v * g.vs + node] * w;
    }
    for (int v = 0; v < 5; ++v) {
        double x = acc[v];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if ((threadIdx.x & 31) == 0) atomicAdd(out + v, x * vol);
    }
}

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------

template <int SCHEME, int FLUX, typename T>
static cudaError_t launch_axis(int axis, const GridView& g, const StageView& sv, cudaStream_t st) {
    if (axis == 0) {
        const int cnt_rows = (g.hi[1] - g.lo[1]) * (g.hi[2] - g.lo[2]);
        dim3 block(32, 4);
        dim3 grid((g.hi[0] - g.lo[0] + 30) / 31, (cnt_rows + 3) / 4, 1);
        sweep_x<SCHEME, FLUX, T><<<grid, block, 0, st>>>(g, sv);
    } else {
        const int other = axis == 1 ? 2 : 1;
        const int segs = (g.hi[axis] - g.lo[axis] + SEGLEN - 1) / SEGLEN;
        dim3 block(32, 4);
        dim3 grid((g.hi[0] - g.lo[0] + 31) / 32, (segs + 3) / 4, g.hi[other] - g.lo[other]);
        if (axis == 1) sweep_yz<1, SCHEME, FLUX, T><<<grid, block, 0, st>>>(g, sv);
        else sweep_yz<2, SCHEME, FLUX, T><<<grid, block, 0, st>>>(g, sv);
    }
    return cudaGetLastError();
}

template <int FLUX, typename T>
static cudaError_t launch_axis_s(int scheme, int axis, const GridView& g, const StageView& sv, cudaStream_t st) {
    switch (scheme) {
    case WENO5: return launch_axis<WENO5, FLUX, T>(axis, g, sv, st);
    case TENO5: return launch_axis<TENO5, FLUX, T>(axis, g, sv, st);
    case WENO3: return launch_axis<WENO3, FLUX, T>(axis, g, sv, st);
    case WENO7: return launch_axis<WENO7, FLUX, T>(axis, g, sv, st);
    }
    return cudaErrorInvalidValue;
}

// Rusanov and Roe in both precisions; Steger-Warming, Lax-Friedrichs and
// Lax-Wendroff faces in FP64.
template <typename T>
static cudaError_t launch_axis_t(int scheme, int flux, int axis, const GridView& g, const StageView& sv,
                                 cudaStream_t st) {
    if (flux == RUSANOV) return launch_axis_s<RUSANOV, T>(scheme, axis, g, sv, st);
    if (flux == ROE) return launch_axis_s<ROE, T>(scheme, axis, g, sv, st);
    if constexpr (sizeof(T) == sizeof(double)) {
        if (flux == STEGER) return launch_axis_s<STEGER, T>(scheme, axis, g, sv, st);
        if (flux == LAXF) return launch_axis_s<LAXF, T>(scheme, axis, g, sv, st);
        if (flux == LAXW) return launch_axis_s<LAXW, T>(scheme, axis, g, sv, st);
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_sweep(int scheme, int flux, int prec64, int axis, const GridView& g, const StageView& sv,
                         cudaStream_t st) {
    return prec64 ? launch_axis_t<double>(scheme, flux, axis, g, sv, st)
                  : launch_axis_t<float>(scheme, flux, axis, g, sv, st);
}

static int grid_for(long long work, int block) {
    long long b = (work + block - 1) / block;
    if (b > 148LL * 16) b = 148LL * 16;
    return (int)(b < 1 ? 1 : b);
}

cudaError_t launch_dt(const GridView& g, const double* q, Clock* clock, unsigned* flags, int skip_if_ready,
                      cudaStream_t st) {
    // one warp per 64-node row chunk (8 chunks per 256-thread block)
    const long long items = (long long)((g.hi[0] - g.lo[0] + 63) / 64) * (g.hi[1] - g.lo[1]) * (g.hi[2] - g.lo[2]);
    dt_kernel<<<grid_for(items * 32, 256), 256, 0, st>>>(g, q, clock, flags, skip_if_ready);
    return cudaGetLastError();
}

cudaError_t launch_finalize_dt(Clock* c, const unsigned* flags, cudaStream_t st) {
    finalize_dt_kernel<<<1, 1, 0, st>>>(c, flags);
    return cudaGetLastError();
}

cudaError_t launch_commit(Clock* c, double* dt_log, long long dt_cap, int cfl_next, cudaStream_t st) {
    commit_kernel<<<1, 1, 0, st>>>(c, dt_log, dt_cap, cfl_next);
    return cudaGetLastError();
}

cudaError_t launch_set_dt(Clock* c, double dt, cudaStream_t st) {
    set_dt_kernel<<<1, 1, 0, st>>>(c, dt);
    return cudaGetLastError();
}

cudaError_t launch_reset_min(Clock* c, cudaStream_t st) {
    reset_min_kernel<<<1, 1, 0, st>>>(c);
    return cudaGetLastError();
}

cudaError_t launch_stage_from_residual(const GridView& g, const StageView& sv, cudaStream_t st) {
    const long long total = (long long)(g.hi[0] - g.lo[0]) * (g.hi[1] - g.lo[1]) * (g.hi[2] - g.lo[2]);
    stage_from_residual_kernel<<<grid_for(total, 256), 256, 0, st>>>(g, sv);
    return cudaGetLastError();
}

cudaError_t launch_aos_to_soa(const double* aos, double* soa, long long nodes, long long vs, cudaStream_t st) {
    aos_to_soa_kernel<<<grid_for((nodes + 127) / 128 * 32, 256), 256, 0, st>>>(aos, soa, nodes, vs);
    return cudaGetLastError();
}

cudaError_t launch_soa_to_aos(const GridView& g, const double* soa, double* aos, cudaStream_t st) {
    const long long items = (long long)((g.n[0] + 127) / 128) * g.n[1] * g.n[2];  // one warp each
    soa_to_aos_kernel<<<grid_for(items * 32, 256), 256, 0, st>>>(g, soa, aos);
    return cudaGetLastError();
}

cudaError_t launch_totals(const GridView& g, const double* q, double* out, double vol, cudaStream_t st) {
    const long long nodes = (long long)g.n[0] * g.n[1] * g.n[2];
    totals_kernel<<<grid_for(nodes, 256), 256, 0, st>>>(g, q, out, vol);
    return cudaGetLastError();
}

}  // namespace sfg
