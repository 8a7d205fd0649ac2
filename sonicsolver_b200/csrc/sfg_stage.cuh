// sfg_stage.cuh -- device helpers shared by the stage kernels: ghost / halo
// index mapping, the stage combination with state validation, status flush.
#pragma once

#include "sfg_internal.h"
#include "sfg_math.cuh"

namespace sfg {

// Ghost and boundary-node values by index mapping (no ghost storage):
// transmissive ends read the inner neighbour (zeroGradient: boundary node <-
// inner node, ghosts <- boundary node; SF_zeroGradient.cpp:88-105), periodic
// ends wrap, frozen ends read the extra end node that holds the frozen ghost
// value.
__device__ __forceinline__ int map_index(int i, int n, int bcl, int bch) {
    if (bcl == BC_PERIODIC) {
        if (i < 0) i += n;
    } else if (bcl == BC_FROZEN) {
        if (i < 0) i = 0;
    } else if (i < 1) {
        i = 1;
    }
    if (bch == BC_PERIODIC) {
        if (i >= n) i -= n;
    } else if (bch == BC_FROZEN) {
        if (i > n - 1) i = n - 1;
    } else if (i > n - 2) {
        i = n - 2;
    }
    return i;
}

// FP32-flux reference state of a stage: the grid's first solved node of the
// stage's input.  Every tile, chunk and segment of a launch takes the same
// one, so a face that two of them evaluate (a tile edge, a chunk boundary)
// gets the same FP32 inputs and the same bits on both sides, and every face
// flux enters the divergence of its two nodes as one value.
__device__ __forceinline__ long long ref_node(const GridView& g) {
    return ((long long)g.lo[2] * g.n[1] + g.lo[1]) * g.n[0] + g.lo[0];
}

// Loads the FP64 reference state of a stage (ref_node of the stage input).
__device__ __forceinline__ void load_ref(const GridView& g, const double* qs, double (&qref)[5]) {
    const long long at = ref_node(g);
#pragma unroll
    for (int v = 0; v < 5; ++v) qref[v] = __ldg(qs + v * g.vs + at);
}

__device__ __forceinline__ void atomic_min_positive(unsigned long long* bits, double v) {
    atomicMin(bits, (unsigned long long)__double_as_longlong(v));
}

// Spectral-radius sum of one node for the CFL step (RusanovEOS::deltaT,
// SF_rusanovEOS.cpp:110-147): sr = sum_active (|u_d| + c) metric_d, with the
// state closed as SingleFluidStateModel::close does (u = m / rho,
// p = (gamma - 1) rho (E - rho |u|^2 / 2) / rho, c = sqrt(gamma p / rho)).
// Every operation is an explicit round-to-nearest intrinsic in the
// reference's order, so the standalone reduction (dt_kernel) and the one fused
// into a step's last stage give the same bits -- and the same bits as the
// oracle's uncontracted C.  dt = CFL / max sr (division is monotonic, so this
// equals the minimum of CFL / sr).
__device__ __forceinline__ double cfl_rate(const GridView& g, const double (&q)[5]) {
    const double rho = q[0];
    const double u = __ddiv_rn(q[1], rho), v = __ddiv_rn(q[2], rho), w = __ddiv_rn(q[3], rho);
    const double uu = __dadd_rn(__dadd_rn(__dmul_rn(u, u), __dmul_rn(v, v)), __dmul_rn(w, w));
    const double kin = __dmul_rn(__dmul_rn(0.5, rho), uu);
    const double e = __ddiv_rn(__dsub_rn(q[4], kin), rho);
    const double p = __dmul_rn(__dmul_rn(g.gamma - 1.0, rho), e);
    const double c = __dsqrt_rn(__ddiv_rn(__dmul_rn(g.gamma, p), rho));
    double sr = __dadd_rn(fabs(__dmul_rn(u, g.metric[0])), __dmul_rn(c, g.metric[0]));
    if (g.dim > 1) sr = __dadd_rn(sr, __dadd_rn(fabs(__dmul_rn(v, g.metric[1])), __dmul_rn(c, g.metric[1])));
    if (g.dim > 2) sr = __dadd_rn(sr, __dadd_rn(fabs(__dmul_rn(w, g.metric[2])), __dmul_rn(c, g.metric[2])));
    return sr;
}

// The same with the node's own metric vectors (curvilinear grids):
// sr = sum_active (|u . m_d| + c |m_d|), in the reference's operation order.
__device__ __forceinline__ double cfl_rate_node(const GridView& g, const double (&q)[5], long long node) {
    if (!g.curv) return cfl_rate(g, q);
    const double rho = q[0];
    const double u = __ddiv_rn(q[1], rho), v = __ddiv_rn(q[2], rho), w = __ddiv_rn(q[3], rho);
    const double uu = __dadd_rn(__dadd_rn(__dmul_rn(u, u), __dmul_rn(v, v)), __dmul_rn(w, w));
    const double kin = __dmul_rn(__dmul_rn(0.5, rho), uu);
    const double e = __ddiv_rn(__dsub_rn(q[4], kin), rho);
    const double p = __dmul_rn(__dmul_rn(g.gamma - 1.0, rho), e);
    const double c = __dsqrt_rn(__ddiv_rn(__dmul_rn(g.gamma, p), rho));
    double sr = 0.0;
    for (int d = 0; d < g.dim; ++d) {
        const double mx = g.node_metric[(3 * d) * g.vs + node], my = g.node_metric[(3 * d + 1) * g.vs + node],
                     mz = g.node_metric[(3 * d + 2) * g.vs + node];
        const double un = fabs(__dadd_rn(__dadd_rn(__dmul_rn(u, mx), __dmul_rn(v, my)), __dmul_rn(w, mz)));
        const double mag = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(mx, mx), __dmul_rn(my, my)), __dmul_rn(mz, mz)));
        sr = __dadd_rn(sr, __dadd_rn(un, __dmul_rn(c, mag)));
    }
    return sr;
}

// Largest sr of a warp, then one atomic: clock->dt_bits = min(.., CFL / sr).
// Callers pass sr = 0 for threads without a node.
__device__ __forceinline__ void flush_cfl_warp(const GridView& g, Clock* clock, double sr) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sr = fmax(sr, __shfl_xor_sync(0xffffffffu, sr, o));
    if ((threadIdx.x & 31) == 0 && sr > 0.0) atomic_min_positive(&clock->dt_bits, __ddiv_rn(g.cfl, sr));
}

// The same for a whole block (every thread of the block must call it).
__device__ __forceinline__ void flush_cfl_block(const GridView& g, Clock* clock, double sr) {
    __shared__ double warp_max[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sr = fmax(sr, __shfl_xor_sync(0xffffffffu, sr, o));
    const int warps = (blockDim.x + 31) >> 5;
    __syncthreads();  // warp_max may still be read by a previous call
    if ((threadIdx.x & 31) == 0) warp_max[threadIdx.x >> 5] = sr;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int i = 1; i < warps; ++i) sr = fmax(sr, warp_max[i]);
        if (sr > 0.0) atomic_min_positive(&clock->dt_bits, __ddiv_rn(g.cfl, sr));
    }
}

// Stage combination at one node for one variable (applySSPStage, applyStage,
// applyFinalRK4, applyDivergence).  qs_v is the current value, r the residual.
__device__ __forceinline__ double stage_value(const StageView& sv, double dt, double qs_v, double r,
                                              long long at) {
    switch (sv.time_id) {
    case T_EULER:
        return qs_v - dt * r;
    case T_SSPRK3: {
        const double euler = qs_v - dt * r;
        return sv.base * sv.q0[at] + sv.inc * euler;
    }
    default: {  // classical RK4 with one accumulator K = k1 + 2 k2 + 2 k3
        if (sv.stage == 0) sv.k[at] = r;
        else if (sv.stage < 3) sv.k[at] = sv.k[at] + 2.0 * r;
        if (sv.stage < 3) return sv.q0[at] - sv.inc * dt * r;
        return sv.q0[at] - dt / 6.0 * (sv.k[at] + 1.0 * r);
    }
    }
}

// Finishes one node: residual output or stage update + state validation
// (validateEquationState after every stage, SF_explicit.cpp:417).  With
// MODE_CFL, sr_max also takes the node's CFL rate of the new state.
// `jac` is the node's 1/J (g.jac on uniform grids); CURV: the CFL rate uses
// the node's metric vectors.
template <bool CURV>
__device__ __forceinline__ void finish_node_j(const GridView& g, const StageView& sv, double dt, long long node,
                                              const double (&qn)[5], double (&div)[5], double jac, unsigned& flags,
                                              double& sr_max) {
    const long long vs = g.vs;
    if (sv.mode & MODE_RESIDUAL) {
#pragma unroll
        for (int v = 0; v < 5; ++v) sv.r[v * vs + node] = jac * div[v];
        return;
    }
    double out[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) out[v] = stage_value(sv, dt, qn[v], jac * div[v] - 0.0, v * vs + node);
#pragma unroll
    for (int v = 0; v < 5; ++v) sv.qout[v * vs + node] = out[v];
    // p = (gamma - 1)(E - |m|^2 / (2 rho)) > 0 with rho > 0 is 2 E rho > |m|^2:
    // the same test without a division (it differs only where p is within
    // rounding of 0)
    const double m2 = out[1] * out[1] + out[2] * out[2] + out[3] * out[3];
    if (!(out[0] > 0.0)) flags |= FLAG_DENSITY;
    else if (!(2.0 * out[4] * out[0] > m2)) flags |= FLAG_PRESSURE;
    if (!isfinite(out[0] + out[1] + out[2] + out[3] + out[4])) flags |= FLAG_NONFINITE;
    if (sv.mode & MODE_CFL) sr_max = fmax(sr_max, CURV ? cfl_rate_node(g, out, node) : cfl_rate(g, out));
}

__device__ __forceinline__ void finish_node(const GridView& g, const StageView& sv, double dt, long long node,
                                            const double (&qn)[5], double (&div)[5], unsigned& flags,
                                            double& sr_max) {
    finish_node_j<false>(g, sv, dt, node, qn, div, g.jac, flags, sr_max);
}

__device__ __forceinline__ void flush_status(const StageView& sv, unsigned flags, unsigned cores, unsigned cut) {
    if (flags) atomicOr(sv.flags, flags);
    if (sv.counters) {
        // one atomic per warp
        unsigned c = cores, k = cut;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            c += __shfl_xor_sync(0xffffffffu, c, o);
            k += __shfl_xor_sync(0xffffffffu, k, o);
        }
        if ((threadIdx.x & 31) == 0 && (c | k)) {
            atomicAdd(sv.counters + 0, (unsigned long long)c);
            atomicAdd(sv.counters + 1, (unsigned long long)k);
        }
    }
}

}  // namespace sfg
