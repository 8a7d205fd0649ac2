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

__device__ __forceinline__ void atomic_min_positive(unsigned long long* bits, double v) {
    atomicMin(bits, (unsigned long long)__double_as_longlong(v));
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
// (validateEquationState after every stage, SF_explicit.cpp:417).
__device__ __forceinline__ void finish_node(const GridView& g, const StageView& sv, double dt, long long node,
                                            const double (&qn)[5], double (&div)[5], unsigned& flags) {
    const long long vs = g.vs;
    if (sv.mode & MODE_RESIDUAL) {
#pragma unroll
        for (int v = 0; v < 5; ++v) sv.r[v * vs + node] = g.jac * div[v];
        return;
    }
    double out[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) out[v] = stage_value(sv, dt, qn[v], g.jac * div[v] - 0.0, v * vs + node);
#pragma unroll
    for (int v = 0; v < 5; ++v) sv.qout[v * vs + node] = out[v];
    const double ke = 0.5 * (out[1] * out[1] + out[2] * out[2] + out[3] * out[3]) / out[0];
    const double p = (g.gamma - 1.0) * (out[4] - ke);
    if (!(out[0] > 0.0)) flags |= FLAG_DENSITY;
    if (!(p > 0.0)) flags |= FLAG_PRESSURE;
    if (!isfinite(out[0] + out[1] + out[2] + out[3] + out[4])) flags |= FLAG_NONFINITE;
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
