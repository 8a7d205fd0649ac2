// sfg_laws.cuh -- the physical boundary laws of one face point of an
// SFG_BC_LAW end (the law arithmetic of sfg_laws.cu), shared by the
// single-grid law kernel and the batched one (sfg_batch.cu).
#pragma once

#include "sfg_internal.h"
#include "sfg_stage.cuh"

namespace sfg {

namespace law_detail {

constexpr double kGasConstant = 287.05;  // makeSingleFluidPerfectGas (fluidStateModel/SF_factory.h:21-33)

__device__ __forceinline__ unsigned state_fault(double rho, double p) {
    if (!isfinite(rho) || !isfinite(p)) return FLAG_NONFINITE;
    return rho > 0.0 ? FLAG_PRESSURE : FLAG_DENSITY;
}

// SingleFluidStateModel::close (SF_singleFluidStateModel.cpp:49-73) with
// PerfectGasEOS::fromDensityEnergy and its checks (SF_perfectGasEOS.h:26-33,
// 80-86): the pressure of q, or a fault bit.
__device__ __forceinline__ unsigned closed_pressure(const double (&q)[5], double gamma, double& p) {
    const double rho = q[0];
    if (!isfinite(rho) || !(rho > 0.0)) return state_fault(rho, 1.0);
    if (!isfinite(q[1]) || !isfinite(q[2]) || !isfinite(q[3])) return FLAG_NONFINITE;
    const double u = __ddiv_rn(q[1], rho), v = __ddiv_rn(q[2], rho), w = __ddiv_rn(q[3], rho);
    const double uu = __dadd_rn(__dadd_rn(__dmul_rn(u, u), __dmul_rn(v, v)), __dmul_rn(w, w));
    const double kin = __dmul_rn(__dmul_rn(0.5, rho), uu);
    const double em = __ddiv_rn(__dsub_rn(q[4], kin), rho);
    const double thermal = __dsub_rn(em, 0.0);
    const double gm1 = __dsub_rn(gamma, 1.0);
    p = __dmul_rn(__dmul_rn(gm1, rho), thermal);
    const double T = __ddiv_rn(__dmul_rn(thermal, gm1), kGasConstant);
    const double c = __dsqrt_rn(__ddiv_rn(__dmul_rn(gamma, p), rho));
    if (!isfinite(em) || !isfinite(p) || !(p > 0.0) || !isfinite(T) || !(T > 0.0) || !isfinite(c) || !(c > 0.0))
        return state_fault(rho, p);
    return 0u;
}

// setEnergyFromPressure (SF_thermodynamicClosure.cpp:166-184) through
// totalEnergyFromPressure / totalEnergyFromThermo
// (SF_singleFluidStateModel.cpp:75-102) and PerfectGasEOS::fromDensityPressure
// (SF_perfectGasEOS.h:43-53): q[4] from the pressure p.
__device__ __forceinline__ unsigned energy_from_pressure(double (&q)[5], double gamma, double p) {
    if (!isfinite(p) || !(p > 0.0)) return state_fault(q[0], p);
    const double rho = q[0];
    if (!isfinite(rho) || !(rho > 0.0)) return state_fault(rho, p);
    if (!isfinite(q[1]) || !isfinite(q[2]) || !isfinite(q[3])) return FLAG_NONFINITE;
    const double gm1 = __dsub_rn(gamma, 1.0);
    const double thermal = __ddiv_rn(p, __dmul_rn(gm1, rho));
    const double e = __dadd_rn(0.0, thermal);
    const double T = __ddiv_rn(p, __dmul_rn(rho, kGasConstant));
    const double c = __dsqrt_rn(__ddiv_rn(__dmul_rn(gamma, p), rho));
    if (!isfinite(e) || !isfinite(T) || !(T > 0.0) || !isfinite(c) || !(c > 0.0)) return state_fault(rho, p);
    const double inv = __ddiv_rn(1.0, rho);
    const double mm = __dadd_rn(__dadd_rn(__dmul_rn(q[1], q[1]), __dmul_rn(q[2], q[2])), __dmul_rn(q[3], q[3]));
    const double kin = __dmul_rn(__dmul_rn(0.5, inv), mm);
    q[4] = __dadd_rn(__dmul_rn(rho, e), kin);
    return 0u;
}

__device__ __forceinline__ void load5(const double* q, long long vs, long long node, double (&out)[5]) {
#pragma unroll
    for (int v = 0; v < 5; ++v) out[v] = q[v * vs + node];
}

}  // namespace law_detail

// Applies the laws to face point t of lv (0 <= t < lv.start[lv.count]):
// writes the boundary node and the end's extra node of q, from the boundary
// node's values before this application in `old`; fault bits go to *flags.
__device__ __forceinline__ void law_fill_point(const GridView& g, const LawView& lv, const double* old, double* q,
                                               long long t, unsigned* flags) {
    using namespace law_detail;
    int e = 0;
    while (t >= lv.start[e + 1]) ++e;
    const int a = lv.axis[e], hi = lv.end[e];
    // face point -> device coordinates (other axes over their solved range)
    long long r = t - lv.start[e];
    int c[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        if (d == a) continue;
        const int span = g.hi[d] - g.lo[d];
        c[d] = g.lo[d] + (int)(r % span);
        r /= span;
    }
    const int n = g.n[a];
    int cb[3] = {c[0], c[1], c[2]}, cs[3] = {c[0], c[1], c[2]}, cx[3] = {c[0], c[1], c[2]};
    cb[a] = hi ? n - 2 : 1;   // boundary node
    cs[a] = hi ? n - 3 : 2;   // inner sample (nearestInsideSample, SF_zeroGradient.cpp:35-52)
    cx[a] = hi ? n - 1 : 0;   // extra node: every ghost layer
    auto lin = [&](const int (&x)[3]) { return ((long long)x[2] * g.n[1] + x[1]) * g.n[0] + x[0]; };
    const long long nb = lin(cb), ns = lin(cs), nx = lin(cx), vs = g.vs;
    double ob[5], og[5], qs[5];
    load5(old, vs, nb, ob);
    load5(old, vs, nx, og);
    load5(q, vs, ns, qs);
    const double gamma = g.gamma;
    double b[5], x[5];
    unsigned fault = 0u;

    // density (FixedValue::applyScalar, SF_fixedValue.cpp:110-127: ghost =
    // 2 v - q_b; ZeroGradient / Symmetry::applyScalar)
    if (lv.rho[e] == LAW_FIXED_VALUE) {
        b[0] = lv.rho_value[e];
        x[0] = __dsub_rn(__dmul_rn(2.0, lv.rho_value[e]), b[0]);
    } else {
        b[0] = qs[0];
        x[0] = b[0];
    }
    // velocity
    const int code = lv.codes[t];
    double p_primed = 0.0;
    if (lv.U[e] == LAW_FIXED_VALUE) {
        // FixedValue::applyVector3 (SF_fixedValue.cpp:129-160)
        const double primed[5] = {b[0], ob[1], ob[2], ob[3], ob[4]};
        fault |= closed_pressure(primed, gamma, p_primed);
#pragma unroll
        for (int d = 0; d < 3; ++d) b[1 + d] = __dmul_rn(b[0], lv.U_value[e][d]);
        const double ghost_cached[5] = {x[0], og[1], og[2], og[3], og[4]};
        double unused;
        fault |= closed_pressure(ghost_cached, gamma, unused);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double u = __ddiv_rn(b[1 + d], b[0]);
            x[1 + d] = __dmul_rn(x[0], __dsub_rn(__dmul_rn(lv.U_value[e][d], 2.0), u));
        }
    } else if (lv.U[e] == LAW_SYMMETRY) {
        // Symmetry::applyVector3 (SF_symmetry.cpp:82-136)
        if (!(isfinite(b[0]) && b[0] > 0.0) || !(isfinite(qs[0]) && qs[0] > 0.0)) fault |= FLAG_DENSITY;
        const double scale = __ddiv_rn(b[0], qs[0]);
#pragma unroll
        for (int d = 0; d < 3; ++d) b[1 + d] = __dmul_rn(qs[1 + d], scale);
        b[1 + a] = 0.0;
        if (!(isfinite(x[0]) && x[0] > 0.0)) fault |= FLAG_DENSITY;
        const double sg = __ddiv_rn(x[0], b[0]);
#pragma unroll
        for (int d = 0; d < 3; ++d) x[1 + d] = __dmul_rn(d == a ? -b[1 + d] : b[1 + d], sg);
    } else {
        // ZeroGradient::applyVector3 (SF_zeroGradient.cpp:107-131)
#pragma unroll
        for (int d = 1; d < 4; ++d) b[d] = x[d] = qs[d];
    }
    // the boundary state the pressure law's cache lookup returns: primed by
    // the velocity law, or cached with the new momentum and the old energy
    // (after an eviction inside the velocity law, or as an edge point's inner
    // sample); fresh otherwise
    bool cached = code != LAW_STATE_FRESH;
    double p_cached = p_primed;
    if (code == LAW_STATE_HALF) {
        const double half[5] = {b[0], b[1], b[2], b[3], ob[4]};
        fault |= closed_pressure(half, gamma, p_cached);
    }
    // pressure (updateEnergyFromPressure, SF_thermodynamicClosure.cpp:219-285)
    double p_ref;
    if (lv.p[e] == LAW_FIXED_VALUE) {
        fault |= energy_from_pressure(b, gamma, lv.p_value[e]);
        if (cached) p_ref = p_cached;
        else fault |= closed_pressure(b, gamma, p_ref);
        fault |= energy_from_pressure(x, gamma, __dsub_rn(__dmul_rn(2.0, lv.p_value[e]), p_ref));
    } else {
        double ps;
        fault |= closed_pressure(qs, gamma, ps);
        fault |= energy_from_pressure(b, gamma, ps);
        if (cached) p_ref = p_cached;
        else fault |= closed_pressure(b, gamma, p_ref);
        fault |= energy_from_pressure(x, gamma, p_ref);
    }
    if (fault) atomicOr(flags, fault);
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        q[v * vs + nb] = b[v];
        q[v * vs + nx] = x[v];
    }
}

}  // namespace sfg
