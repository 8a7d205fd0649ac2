// sfg_curv.cu -- the stage operator on curvilinear grids: per-node metrics
// (Jac = 1/J and the xi / eta / zeta vectors the reference Field carries,
// src/infrastructure/mesh/SF_mesh.cpp:260-339) and per-face geometry
// (canonicalFace::geometry, methods/numerics/structured/SF_canonicalFace.h:56-118).
//
//   curv_geometry_kernel  once per sfg_set_metrics: for every face (i | i+1)
//                         the cofactor 0.5 (m_i / Jac_i + m_i+1 / Jac_i+1),
//                         its magnitude (the area) and the unit normal,
//                         stored at the lower node i (4 x vs per axis).
//   curv_face_kernel      per axis and stage: one thread per face; the
//                         characteristic reconstruction with the full 5 x 5
//                         left / right eigenvectors of the face normal
//                         (Riemann::buildCharacteristicMatrix,
//                         convection/SF_riemann.cpp:69-123), the face flux
//                         along that normal, times the area.
//   curv_stage_kernel     per stage: R = Jac_node * sum_d (F_d[i] - F_d[i-1])
//                         and the stage update.
//
// FP64.  Reads per node and stage: the state (stencils, mostly from L2), 4
// doubles of face geometry per axis, Jac; writes 5 face fluxes per axis.
#include <algorithm>
#include <type_traits>

#include "sfg_internal.h"
#include "sfg_stage.cuh"
#include "sfg_tile.cuh"

namespace sfg {

namespace {

// physical_pressure with the validity bits (requirePhysicalState).
__device__ __forceinline__ double pressure_n(const double (&q)[5], double gamma, unsigned& flags) {
    if (!isfinite(q[0] + q[1] + q[2] + q[3] + q[4])) flags |= FLAG_NONFINITE;
    if (!(q[0] > 0.0)) flags |= FLAG_DENSITY;
    const double inv = 1.0 / q[0];
    const double ke = 0.5 * (q[1] * q[1] + q[2] * q[2] + q[3] * q[3]) * inv;
    const double p = (gamma - 1.0) * (q[4] - ke);
    if (!(p > 0.0)) flags |= FLAG_PRESSURE;
    return p;
}

// Left / right eigenvectors of the flux Jacobian along the unit normal n
// (Riemann::buildCharacteristicMatrix, SF_riemann.cpp:69-123): tangents l, m
// from n, acoustic rows with the (gamma - 1)|u|^2 / (4 c^2) kinetic term.
__device__ __forceinline__ void char_matrix_n(const double (&q)[5], const double (&n)[3], double gamma,
                                              double (&L)[5][5], double (&R)[5][5], unsigned& flags) {
    const double p = pressure_n(q, gamma, flags);
    const double invR = 1.0 / q[0];
    const double u = q[1] * invR, v = q[2] * invR, w = q[3] * invR;
    const double q2 = u * u + v * v + w * w;
    const double c = sqrt(gamma * p * invR);
    const double H = (q[4] + p) * invR;
    const double n1 = n[0], n2 = n[1], n3 = n[2];
    double l1, l2, l3;
    if (fabs(n3) <= fabs(n2)) {
        const double ss = sqrt(n1 * n1 + n2 * n2);
        l1 = -n2 / ss;
        l2 = n1 / ss;
        l3 = 0.0;
    } else {
        const double ss = sqrt(n1 * n1 + n3 * n3);
        l1 = -n3 / ss;
        l2 = 0.0;
        l3 = n1 / ss;
    }
    const double m1 = n2 * l3 - n3 * l2, m2 = n3 * l1 - n1 * l3, m3 = n1 * l2 - n2 * l1;
    const double un = u * n1 + v * n2 + w * n3;
    const double ul = u * l1 + v * l2 + w * l3;
    const double um = u * m1 + v * m2 + w * m3;
    const double b1 = (gamma - 1.0) / (c * c);
    const double b2 = 0.5 * b1;
    const double x1 = 1.0 / (2.0 * c);
    const double Lm[5][5] = {{1.0 - b2 * q2, b1 * u, b1 * v, b1 * w, -b1},
                             {-ul, l1, l2, l3, 0.0},
                             {-um, m1, m2, m3, 0.0},
                             {0.5 * b2 * q2 + x1 * un, -x1 * n1 - b2 * u, -x1 * n2 - b2 * v, -x1 * n3 - b2 * w, b2},
                             {0.5 * b2 * q2 - x1 * un, x1 * n1 - b2 * u, x1 * n2 - b2 * v, x1 * n3 - b2 * w, b2}};
    const double Rm[5][5] = {{1.0, 0.0, 0.0, 1.0, 1.0},
                             {u, l1, m1, u - c * n1, u + c * n1},
                             {v, l2, m2, v - c * n2, v + c * n2},
                             {w, l3, m3, w - c * n3, w + c * n3},
                             {0.5 * q2, ul, um, H - c * un, H + c * un}};
#pragma unroll
    for (int r = 0; r < 5; ++r)
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            L[r][k] = Lm[r][k];
            R[r][k] = Rm[r][k];
        }
}

// The same eigen-structure held as its basis scalars: row k of L and column k
// of R are formed when field k is reconstructed, so the face kernel keeps
// ~20 values live instead of two 5 x 5 matrices.
template <typename T>
struct CharBasisT {
    T u, v, w, c, H, q2, n1, n2, n3, l1, l2, l3, m1, m2, m3, un, ul, um, b1, b2, x1;
};
using CharBasis = CharBasisT<double>;

// The basis of the state q with pressure p along the unit normal n.
template <typename T>
__device__ __forceinline__ void char_basis_p(const T (&q)[5], T p, const T (&n)[3], T gamma, CharBasisT<T>& e) {
    const T one = T(1), half = T(0.5);
    const T invR = one / q[0];
    e.u = q[1] * invR;
    e.v = q[2] * invR;
    e.w = q[3] * invR;
    e.q2 = e.u * e.u + e.v * e.v + e.w * e.w;
    e.c = sqrt_<T>(gamma * p * invR);
    e.H = (q[4] + p) * invR;
    e.n1 = n[0];
    e.n2 = n[1];
    e.n3 = n[2];
    if (fabs(e.n3) <= fabs(e.n2)) {
        const T ss = sqrt_<T>(e.n1 * e.n1 + e.n2 * e.n2);
        e.l1 = -e.n2 / ss;
        e.l2 = e.n1 / ss;
        e.l3 = T(0);
    } else {
        const T ss = sqrt_<T>(e.n1 * e.n1 + e.n3 * e.n3);
        e.l1 = -e.n3 / ss;
        e.l2 = T(0);
        e.l3 = e.n1 / ss;
    }
    e.m1 = e.n2 * e.l3 - e.n3 * e.l2;
    e.m2 = e.n3 * e.l1 - e.n1 * e.l3;
    e.m3 = e.n1 * e.l2 - e.n2 * e.l1;
    e.un = e.u * e.n1 + e.v * e.n2 + e.w * e.n3;
    e.ul = e.u * e.l1 + e.v * e.l2 + e.w * e.l3;
    e.um = e.u * e.m1 + e.v * e.m2 + e.w * e.m3;
    e.b1 = (gamma - one) / (e.c * e.c);
    e.b2 = half * e.b1;
    e.x1 = one / (T(2) * e.c);
}

__device__ __forceinline__ void char_basis_n(const double (&q)[5], const double (&n)[3], double gamma, CharBasis& e,
                                             unsigned& flags) {
    char_basis_p<double>(q, pressure_n(q, gamma, flags), n, gamma, e);
}

// Row K of L (as char_matrix_n builds it).
template <int K, typename T>
__device__ __forceinline__ void left_row(const CharBasisT<T>& e, T (&r)[5]) {
    const T half = T(0.5), zero = T(0), one = T(1);
    if constexpr (K == 0) {
        r[0] = one - e.b2 * e.q2; r[1] = e.b1 * e.u; r[2] = e.b1 * e.v; r[3] = e.b1 * e.w; r[4] = -e.b1;
    } else if constexpr (K == 1) {
        r[0] = -e.ul; r[1] = e.l1; r[2] = e.l2; r[3] = e.l3; r[4] = zero;
    } else if constexpr (K == 2) {
        r[0] = -e.um; r[1] = e.m1; r[2] = e.m2; r[3] = e.m3; r[4] = zero;
    } else if constexpr (K == 3) {
        r[0] = half * e.b2 * e.q2 + e.x1 * e.un; r[1] = -e.x1 * e.n1 - e.b2 * e.u;
        r[2] = -e.x1 * e.n2 - e.b2 * e.v; r[3] = -e.x1 * e.n3 - e.b2 * e.w; r[4] = e.b2;
    } else {
        r[0] = half * e.b2 * e.q2 - e.x1 * e.un; r[1] = e.x1 * e.n1 - e.b2 * e.u;
        r[2] = e.x1 * e.n2 - e.b2 * e.v; r[3] = e.x1 * e.n3 - e.b2 * e.w; r[4] = e.b2;
    }
}

// Column K of R.
template <int K, typename T>
__device__ __forceinline__ void right_col(const CharBasisT<T>& e, T (&r)[5]) {
    const T half = T(0.5), zero = T(0), one = T(1);
    if constexpr (K == 0) {
        r[0] = one; r[1] = e.u; r[2] = e.v; r[3] = e.w; r[4] = half * e.q2;
    } else if constexpr (K == 1) {
        r[0] = zero; r[1] = e.l1; r[2] = e.l2; r[3] = e.l3; r[4] = e.ul;
    } else if constexpr (K == 2) {
        r[0] = zero; r[1] = e.m1; r[2] = e.m2; r[3] = e.m3; r[4] = e.um;
    } else if constexpr (K == 3) {
        r[0] = one; r[1] = e.u - e.c * e.n1; r[2] = e.v - e.c * e.n2; r[3] = e.w - e.c * e.n3; r[4] = e.H - e.c * e.un;
    } else {
        r[0] = one; r[1] = e.u + e.c * e.n1; r[2] = e.v + e.c * e.n2; r[3] = e.w + e.c * e.n3; r[4] = e.H + e.c * e.un;
    }
}

// Field K of the characteristic reconstruction: project the stencil on row
// K, reconstruct both sides, add column K times the results to qL / qR.
template <int K, int SCHEME, int NST, int W, typename T>
__device__ __forceinline__ void recon_field(const CharBasisT<T>& e, const T (&st)[NST][5], T (&qL)[5], T (&qR)[5],
                                            unsigned& flags, unsigned& cut) {
    T row[5];
    left_row<K, T>(e, row);
    T ch[NST];
#pragma unroll
    for (int s = 0; s < NST; ++s) {
        T acc = T(0);
#pragma unroll
        for (int k = 0; k < 5; ++k) acc += row[k] * st[s][k];
        ch[s] = acc;
    }
    T wl, wr;
    if constexpr (std::is_same<T, float>::value && (SCHEME == WENO5 || SCHEME == TENO5)) {
        // FP32 WENO5 / TENO5: the left- and right-biased stencils as the two
        // lanes of one paired core (the Cartesian kernels' cores)
        float2 v[5];
#pragma unroll
        for (int s = 0; s < 5; ++s) v[s] = make_float2(ch[s], ch[NST - 1 - s]);
        float2 bad = f2(0.f), kept = f2(0.f);
        float2 w;
        if constexpr (SCHEME == TENO5) {
            w = teno5_core2(v, bad, true, kept);
            cut += 6u - unsigned(kept.x + kept.y);
        } else {
            w = weno5_core2(v, bad);
        }
        flag_bad(bad, flags);
        wl = w.x;
        wr = w.y;
    } else {
        T sl[8], sr[8];
#pragma unroll
        for (int s = 0; s < W; ++s) {
            sl[s] = ch[s];
            sr[s] = ch[NST - 1 - s];
        }
        wl = recon_core<SCHEME, T>(sl, flags, cut);
        wr = recon_core<SCHEME, T>(sr, flags, cut);
    }
    T col[5];
    right_col<K, T>(e, col);
#pragma unroll
    for (int r = 0; r < 5; ++r) {
        qL[r] += col[r] * wl;
        qR[r] += col[r] * wr;
    }
}

__device__ __forceinline__ void gemv5(const double (&M)[5][5], const double (&x)[5], double (&y)[5]) {
#pragma unroll
    for (int r = 0; r < 5; ++r) {
        double acc = 0.0;
#pragma unroll
        for (int k = 0; k < 5; ++k) acc += M[r][k] * x[k];
        y[r] = acc;
    }
}

// Physical flux along n (Euler flux of one state).
__device__ __forceinline__ void euler_flux_n(const double (&q)[5], const double (&n)[3], double gamma,
                                             double (&f)[5], unsigned& flags) {
    const double p = pressure_n(q, gamma, flags);
    const double rho = q[0];
    const double u = q[1] / rho, v = q[2] / rho, w = q[3] / rho;
    const double un = u * n[0] + v * n[1] + w * n[2];
    f[0] = rho * un;
    f[1] = rho * u * un + p * n[0];
    f[2] = rho * v * un + p * n[1];
    f[3] = rho * w * un + p * n[2];
    f[4] = (q[4] + p) * un;
}

// Rusanov with both sides closed (RusanovEOS::faceFlux, SF_rusanovEOS.cpp:47-77).
__device__ __forceinline__ void rusanov_n(const double (&qL)[5], const double (&qR)[5], const double (&n)[3],
                                          double gamma, double (&F)[5], unsigned& flags) {
    const double iL = 1.0 / qL[0], iR = 1.0 / qR[0];
    const double uL[3] = {qL[1] * iL, qL[2] * iL, qL[3] * iL}, uR[3] = {qR[1] * iR, qR[2] * iR, qR[3] * iR};
    const double eL = (qL[4] - 0.5 * qL[0] * (uL[0] * uL[0] + uL[1] * uL[1] + uL[2] * uL[2])) / qL[0];
    const double eR = (qR[4] - 0.5 * qR[0] * (uR[0] * uR[0] + uR[1] * uR[1] + uR[2] * uR[2])) / qR[0];
    const double pL = (gamma - 1.0) * qL[0] * eL, pR = (gamma - 1.0) * qR[0] * eR;
    if (!(qL[0] > 0.0) || !(qR[0] > 0.0)) flags |= FLAG_DENSITY;
    if (!(pL > 0.0) || !(pR > 0.0)) flags |= FLAG_PRESSURE;
    const double cL = sqrt(gamma * pL / qL[0]), cR = sqrt(gamma * pR / qR[0]);
    const double unL = uL[0] * n[0] + uL[1] * n[1] + uL[2] * n[2];
    const double unR = uR[0] * n[0] + uR[1] * n[1] + uR[2] * n[2];
    double fL[5], fR[5];
    fL[0] = qL[0] * unL;
    fR[0] = qR[0] * unR;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        fL[1 + d] = qL[1 + d] * unL + pL * n[d];
        fR[1 + d] = qR[1 + d] * unR + pR * n[d];
    }
    fL[4] = (qL[4] + pL) * unL;
    fR[4] = (qR[4] + pR) * unR;
    const double lam = fmax(fabs(unL) + cL, fabs(unR) + cR);
    if (!isfinite(lam) || !(lam > 0.0)) flags |= FLAG_NONFINITE;
#pragma unroll
    for (int k = 0; k < 5; ++k) F[k] = 0.5 * (fL[k] + fR[k]) - 0.5 * lam * (qR[k] - qL[k]);
}

// Roe with the entropy fix and the reference's eigenvalue / eigenvector
// pairing (Flux::RoeFlux::flux, SF_roe.cpp:10-90).
__device__ __forceinline__ void roe_n(const double (&qL)[5], const double (&qR)[5], const double (&n)[3],
                                      double gamma, double (&F)[5], unsigned& flags) {
    const double gm1 = gamma - 1.0;
    const double pL = pressure_n(qL, gamma, flags), pR = pressure_n(qR, gamma, flags);
    const double iL = 1.0 / qL[0], iR = 1.0 / qR[0];
    const double uL = qL[1] * iL, vL = qL[2] * iL, wL = qL[3] * iL, hL = (qL[4] + pL) * iL;
    const double uR = qR[1] * iR, vR = qR[2] * iR, wR = qR[3] * iR, hR = (qR[4] + pR) * iR;
    const double sL = sqrt(qL[0]), sR = sqrt(qR[0]), ss = sL + sR;
    const double ur = (sL * uL + sR * uR) / ss, vr = (sL * vL + sR * vR) / ss, wr = (sL * wL + sR * wR) / ss;
    const double hr = (sL * hL + sR * hR) / ss;
    const double q2 = ur * ur + vr * vr + wr * wr;
    const double a2 = gm1 * (hr - 0.5 * q2);
    if (!isfinite(a2) || !(a2 > 0.0)) flags |= FLAG_ROE_SOUND;
    const double a = sqrt(a2);
    const double unr = ur * n[0] + vr * n[1] + wr * n[2];
    const double lam[5] = {unr, unr, unr, unr + a, unr - a};
    const double eps = 0.1 * a;
    double al[5];
#pragma unroll
    for (int m = 0; m < 5; ++m) {
        const double x = fabs(lam[m]);
        al[m] = x < 2.0 * eps ? 0.5 * (x * x / (2.0 * eps) + eps) : x;
    }
    const double rr = sL * sR;
    const double qRoe[5] = {rr, rr * ur, rr * vr, rr * wr, rr * (0.5 * q2 + a2 / gm1)};
    double L[5][5], R[5][5];
    char_matrix_n(qRoe, n, gamma, L, R, flags);
    double dQ[5], alpha[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) dQ[k] = qR[k] - qL[k];
    gemv5(L, dQ, alpha);
    double diss[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int wv = 0; wv < 5; ++wv) {
        const double strength = al[wv] * alpha[wv];
#pragma unroll
        for (int k = 0; k < 5; ++k) diss[k] += R[k][wv] * strength;
    }
    double fL[5], fR[5];
    euler_flux_n(qL, n, gamma, fL, flags);
    euler_flux_n(qR, n, gamma, fR, flags);
#pragma unroll
    for (int k = 0; k < 5; ++k) F[k] = 0.5 * (fL[k] + fR[k] - diss[k]);
}

// Steger-Warming split of one state (Flux::StegerWarmingFlux, SF_sw.cpp),
// entropy-fixed eigenvalue parts; POS: the positive part.
template <bool POS>
__device__ __forceinline__ void steger_part_n(const double (&q)[5], const double (&n)[3], double gamma,
                                              double (&f)[5], unsigned& flags) {
    const double p = pressure_n(q, gamma, flags);
    const double r = q[0], invR = 1.0 / r;
    const double u = q[1] * invR, v = q[2] * invR, w = q[3] * invR;
    const double q2 = u * u + v * v + w * w;
    const double a = sqrt(gamma * p * invR);
    const double un = u * n[0] + v * n[1] + w * n[2];
    const double lam[5] = {un, un, un, un + a, un - a};
    double l[5];
    const double eps = 0.01;
#pragma unroll
    for (int i = 0; i < 5; ++i) {
        double lp, lm;
        if (fabs(lam[i]) < 2.0 * eps) {
            lp = 0.5 * (lam[i] * lam[i] / (4.0 * eps) + lam[i] + eps);
            lm = lam[i] - lp;
        } else {
            lp = 0.5 * (lam[i] + fabs(lam[i]));
            lm = 0.5 * (lam[i] - fabs(lam[i]));
        }
        l[i] = POS ? lp : lm;
    }
    const double common = r / (2.0 * gamma);
    const double W1 = 2.0 * (gamma - 1.0) * l[0] + l[3] + l[4], W2 = l[3] - l[4], W3 = l[3] + l[4];
    f[0] = common * W1;
    f[1] = common * (u * W1 + a * n[0] * W2);
    f[2] = common * (v * W1 + a * n[1] * W2);
    f[3] = common * (w * W1 + a * n[2] * W2);
    f[4] = common * (0.5 * q2 * W1 + a * un * W2 + (a * a / (gamma - 1.0)) * W3);
}

// Local Lax-Friedrichs split of one state (Flux::LaxFriedrichsFlux, SF_lxF.cpp).
__device__ __forceinline__ void laxf_part_n(const double (&q)[5], const double (&n)[3], double gamma, double sign,
                                            double (&f)[5], unsigned& flags) {
    const double p = pressure_n(q, gamma, flags);
    const double r = q[0], invR = 1.0 / r;
    const double u = q[1] * invR, v = q[2] * invR, w = q[3] * invR;
    const double a = sqrt(gamma * p * invR);
    const double un = u * n[0] + v * n[1] + w * n[2];
    const double lam = fabs(un) + a;
    const double Fp[5] = {r * un, q[1] * un + p * n[0], q[2] * un + p * n[1], q[3] * un + p * n[2], (q[4] + p) * un};
#pragma unroll
    for (int i = 0; i < 5; ++i) f[i] = 0.5 * (Fp[i] + sign * lam * q[i]);
}

template <int FLUX>
__device__ __forceinline__ void flux_n(const double (&qL)[5], const double (&qR)[5], const double (&n)[3],
                                       double gamma, double (&F)[5], unsigned& flags) {
    if constexpr (FLUX == RUSANOV) {
        rusanov_n(qL, qR, n, gamma, F, flags);
    } else if constexpr (FLUX == ROE) {
        roe_n(qL, qR, n, gamma, F, flags);
    } else if constexpr (FLUX == STEGER) {
        double fp[5], fm[5];
        steger_part_n<true>(qL, n, gamma, fp, flags);
        steger_part_n<false>(qR, n, gamma, fm, flags);
#pragma unroll
        for (int k = 0; k < 5; ++k) F[k] = fp[k] + fm[k];
    } else {
        double fp[5], fm[5];
        laxf_part_n(qL, n, gamma, 1.0, fp, flags);
        laxf_part_n(qR, n, gamma, -1.0, fm, flags);
#pragma unroll
        for (int k = 0; k < 5; ++k) F[k] = fp[k] + fm[k];
    }
}

// ---- FP32-flux form -------------------------------------------------------
// A face's stencil as FP32 deviations d = q - q_ref from its left node q_ref
// (FP64); the reconstruction runs on the deviations (projections are linear,
// the WENO / TENO cores shift invariant) and the face flux comes back as the
// deviation F(q) - F(q_ref) in algebra that never subtracts large terms; the
// FP64 flux of q_ref along the face normal is added in FP64.

// Physical flux along the unit normal n of q = q_ref + d, as the deviation
// F(q) - F(q_ref):
//   du = (d_m - u_ref d_rho) / rho,  dp = (gamma - 1)(d_E - (m_ref.du + d_m.u) / 2)
//   dF_rho = d_m.n,  dF_m = m_ref du_n + d_m u_n + dp n,  dF_E = (E_ref + p_ref) du_n + (d_E + dp) u_n.
__device__ __forceinline__ void phys_flux_dev_n(const Ref32& r, const float (&d)[5], const float (&n)[3], float gamma,
                                                float (&F)[5], float& un, float& c, float& p_out, unsigned& flags) {
    const float rho = r.q[0] + d[0];
    const float irho = rcp_approx(rho);
    float du[3], u[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        du[k] = (d[1 + k] - r.u[k] * d[0]) * irho;
        u[k] = r.u[k] + du[k];
    }
    const float dmu = r.q[1] * du[0] + r.q[2] * du[1] + r.q[3] * du[2] + d[1] * u[0] + d[2] * u[1] + d[3] * u[2];
    const float dp = (gamma - 1.f) * (d[4] - 0.5f * dmu);
    const float p = r.p + dp;
    if (!(rho > 0.f)) flags |= FLAG_DENSITY;
    if (!(p > 0.f)) flags |= FLAG_PRESSURE;
    const float dun = du[0] * n[0] + du[1] * n[1] + du[2] * n[2];
    un = u[0] * n[0] + u[1] * n[1] + u[2] * n[2];
    F[0] = d[1] * n[0] + d[2] * n[1] + d[3] * n[2];
#pragma unroll
    for (int k = 0; k < 3; ++k) F[1 + k] = r.q[1 + k] * dun + d[1 + k] * un + dp * n[k];
    F[4] = (r.q[4] + r.p) * dun + (d[4] + dp) * un;
    c = sqrtf(gamma * p * irho);
    p_out = p;
}

template <int FLUX>
__device__ __forceinline__ void flux_dev_n(const Ref32& r, const float (&dL)[5], const float (&dR)[5],
                                           const float (&n)[3], float gamma, float (&F)[5], unsigned& flags) {
    float fL[5], fR[5], unL, unR, cL, cR, pL, pR;
    phys_flux_dev_n(r, dL, n, gamma, fL, unL, cL, pL, flags);
    phys_flux_dev_n(r, dR, n, gamma, fR, unR, cR, pR, flags);
    if constexpr (FLUX == RUSANOV) {
        const float hl = 0.5f * fmaxf(fabsf(unL) + cL, fabsf(unR) + cR);
#pragma unroll
        for (int v = 0; v < 5; ++v) F[v] = 0.5f * (fL[v] + fR[v]) - hl * (dR[v] - dL[v]);
    } else {
        // Roe: average and eigen-structure from the absolute states, the
        // dissipation from the jump dR - dL (SF_roe.cpp:10-90)
        float qL[5], qR[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            qL[v] = r.q[v] + dL[v];
            qR[v] = r.q[v] + dR[v];
        }
        const float gm1 = gamma - 1.f;
        const float iL = rcp_approx(qL[0]), iR = rcp_approx(qR[0]);
        const float hL = (qL[4] + pL) * iL, hR = (qR[4] + pR) * iR;
        const float sL = sqrtf(qL[0]), sR = sqrtf(qR[0]);
        const float iS = rcp_approx(sL + sR);
        const float ur = (sL * qL[1] * iL + sR * qR[1] * iR) * iS;
        const float vr = (sL * qL[2] * iL + sR * qR[2] * iR) * iS;
        const float wr = (sL * qL[3] * iL + sR * qR[3] * iR) * iS;
        const float hr = (sL * hL + sR * hR) * iS;
        const float q2 = ur * ur + vr * vr + wr * wr;
        const float a2 = gm1 * (hr - 0.5f * q2);
        if (!(a2 > 0.f) || !isfinite(a2)) flags |= FLAG_ROE_SOUND;
        const float rr = sL * sR;
        const float qRoe[5] = {rr, rr * ur, rr * vr, rr * wr, rr * (0.5f * q2 + __fdividef(a2, gm1))};
        // the Roe state's own pressure, (gamma - 1)(E - rho q2 / 2) = rho a2, as
        // the FP64 path closes it for the eigenvectors
        CharBasisT<float> e;
        char_basis_p<float>(qRoe, rr * a2, n, gamma, e);
        const float a = sqrtf(a2);
        const float unr = ur * n[0] + vr * n[1] + wr * n[2];
        const float lam[5] = {unr, unr, unr, unr + a, unr - a};
        const float delta = 0.1f * a;
        float dq[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) dq[v] = dR[v] - dL[v];
        float diss[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
        auto wave = [&](auto kc) {
            constexpr int K = decltype(kc)::value;
            float row[5], col[5];
            left_row<K, float>(e, row);
            right_col<K, float>(e, col);
            const float alpha = row[0] * dq[0] + row[1] * dq[1] + row[2] * dq[2] + row[3] * dq[3] + row[4] * dq[4];
            const float val = fabsf(lam[K]);
            const float ab = val < 2.f * delta ? 0.5f * (val * val * rcp_approx(2.f * delta) + delta) : val;
#pragma unroll
            for (int v = 0; v < 5; ++v) diss[v] += col[v] * (ab * alpha);
        };
        wave(std::integral_constant<int, 0>{});
        wave(std::integral_constant<int, 1>{});
        wave(std::integral_constant<int, 2>{});
        wave(std::integral_constant<int, 3>{});
        wave(std::integral_constant<int, 4>{});
#pragma unroll
        for (int v = 0; v < 5; ++v) F[v] = 0.5f * (fL[v] + fR[v] - diss[v]);
    }
}

// One face in the FP32-flux form: stencil deviations d from the reference
// ref, eigen basis at the face average, characteristic reconstruction, flux
// deviation along the unit normal n (per unit area).
template <int SCHEME, int FLUX>
__device__ __forceinline__ void curv_face_dev32(const float (&d)[SchemeInfo<SCHEME>::NST][5], const Ref32& ref,
                                                const float (&n)[3], float gamma, float (&F)[5], unsigned& flags,
                                                unsigned& cut) {
    constexpr int NST = SchemeInfo<SCHEME>::NST, W = SchemeInfo<SCHEME>::W, CL = NST / 2 - 1;
    float qa[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) qa[v] = ref.q[v] + 0.5f * (d[CL][v] + d[CL + 1][v]);
    const float pa = (gamma - 1.f) * (qa[4] - 0.5f * (qa[1] * qa[1] + qa[2] * qa[2] + qa[3] * qa[3]) / qa[0]);
    if (!(qa[0] > 0.f) || !(pa > 0.f)) flags |= FLAG_PRESSURE;
    CharBasisT<float> e;
    char_basis_p<float>(qa, pa, n, gamma, e);
    float dL[5] = {0.f, 0.f, 0.f, 0.f, 0.f}, dR[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
    recon_field<0, SCHEME, NST, W, float>(e, d, dL, dR, flags, cut);
    recon_field<1, SCHEME, NST, W, float>(e, d, dL, dR, flags, cut);
    recon_field<2, SCHEME, NST, W, float>(e, d, dL, dR, flags, cut);
    recon_field<3, SCHEME, NST, W, float>(e, d, dL, dR, flags, cut);
    recon_field<4, SCHEME, NST, W, float>(e, d, dL, dR, flags, cut);
    flux_dev_n<FLUX>(ref, dL, dR, n, gamma, F, flags);
}

}  // namespace

// ---------------------------------------------------------------------------
// Face geometry from node metrics (SF_canonicalFace.h:56-118): stored for the
// faces whose lower node is i; the upper node wraps on periodic axes and
// does not exist past the last node of other axes (nothing stored).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) curv_geometry_kernel(GridView g, const double* __restrict__ nm,
                                                            double* geom0, double* geom1, double* geom2,
                                                            unsigned* flags) {
    const long long nodes = (long long)g.n[0] * g.n[1] * g.n[2];
    const long long vs = g.vs;
    double* geom[3] = {geom0, geom1, geom2};
    unsigned fl = 0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nodes;
         t += (long long)gridDim.x * blockDim.x) {
        const int c[3] = {(int)(t % g.n[0]), (int)((t / g.n[0]) % g.n[1]), (int)(t / ((long long)g.n[0] * g.n[1]))};
        for (int a = 0; a < g.dim; ++a) {
            int cu[3] = {c[0], c[1], c[2]};
            cu[a] = c[a] + 1;
            if (cu[a] >= g.n[a]) {
                if (g.bc_hi[a] != BC_PERIODIC) continue;
                cu[a] = 0;
            }
            const long long up = ((long long)cu[2] * g.n[1] + cu[1]) * g.n[0] + cu[0];
            const double ja = nm[t], jb = nm[up];
            if (!isfinite(ja) || !isfinite(jb) || fabs(ja) < 1.0e-30 || fabs(jb) < 1.0e-30) fl |= FLAG_NONFINITE;
            double cof[3];
#pragma unroll
            for (int k = 0; k < 3; ++k)
                cof[k] = 0.5 * (__ddiv_rn(nm[(1 + 3 * a + k) * vs + t], ja) + __ddiv_rn(nm[(1 + 3 * a + k) * vs + up], jb));
            const double area = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(cof[0], cof[0]), __dmul_rn(cof[1], cof[1])),
                                                     __dmul_rn(cof[2], cof[2])));
            if (!isfinite(area) || !(area > 0.0)) fl |= FLAG_NONFINITE;
#pragma unroll
            for (int k = 0; k < 3; ++k) geom[a][k * vs + t] = __ddiv_rn(cof[k], area);
            geom[a][3 * vs + t] = area;
        }
    }
    if (fl) atomicOr(flags, fl);
}

// ---------------------------------------------------------------------------
// Face fluxes along one axis.  Faces: lower node over [lo - 1, hi - 1] on a
// bounded axis, [0, n) on a periodic one; the other axes over the solved
// range.  F (times the face area) goes to fl[axis][v] at the lower node.
// ---------------------------------------------------------------------------
template <int SCHEME, int FLUX>
__global__ void __launch_bounds__(128, 4) curv_face_kernel(GridView g, StageView sv, int axis, double* fl) {
    if (sv.require_active && !sv.clock->active) return;
    constexpr int NST = SchemeInfo<SCHEME>::NST, W = SchemeInfo<SCHEME>::W;
    const int a = axis;
    int base[3], span[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const bool per = d < g.dim && g.bc_lo[d] == BC_PERIODIC;
        base[d] = d == a ? (per ? 0 : g.lo[d] - 1) : g.lo[d];
        span[d] = d == a ? (per ? g.n[d] : g.hi[d] - g.lo[d] + 1) : g.hi[d] - g.lo[d];
    }
    const long long total = (long long)span[0] * span[1] * span[2];
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    unsigned flags = 0, cut = 0, cores = 0;
    if (t < total) {
        int c[3];
        long long r = t;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            c[d] = base[d] + (int)(r % span[d]);
            r /= span[d];
        }
        const long long vs = g.vs;
        double st[NST][5];
#pragma unroll
        for (int s = 0; s < NST; ++s) {
            int cc[3] = {c[0], c[1], c[2]};
            cc[a] = map_index(c[a] - (NST / 2 - 1) + s, g.n[a], g.bc_lo[a], g.bc_hi[a]);
            const long long node = ((long long)cc[2] * g.n[1] + cc[1]) * g.n[0] + cc[0];
#pragma unroll
            for (int v = 0; v < 5; ++v) st[s][v] = sv.qs[v * vs + node];
        }
        const long long face = ((long long)c[2] * g.n[1] + c[1]) * g.n[0] + c[0];
        const double* gm = g.geom[a];
        const double n[3] = {gm[face], gm[vs + face], gm[2 * vs + face]};
        const double area = gm[3 * vs + face];
        double qavg[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) qavg[v] = 0.5 * (st[NST / 2 - 1][v] + st[NST / 2][v]);
        CharBasis e;
        char_basis_n(qavg, n, g.gamma, e, flags);
        double qL[5] = {0.0, 0.0, 0.0, 0.0, 0.0}, qR[5] = {0.0, 0.0, 0.0, 0.0, 0.0}, F[5];
        recon_field<0, SCHEME, NST, W>(e, st, qL, qR, flags, cut);
        recon_field<1, SCHEME, NST, W>(e, st, qL, qR, flags, cut);
        recon_field<2, SCHEME, NST, W>(e, st, qL, qR, flags, cut);
        recon_field<3, SCHEME, NST, W>(e, st, qL, qR, flags, cut);
        recon_field<4, SCHEME, NST, W>(e, st, qL, qR, flags, cut);
        if (SCHEME == TENO5) cores += 10;
        flux_n<FLUX>(qL, qR, n, g.gamma, F, flags);
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            const double x = F[v] * area;
            if (!isfinite(x)) flags |= FLAG_NONFINITE;
            fl[((long long)a * 5 + v) * vs + face] = x;
        }
    }
    flush_status(sv, flags, cores, cut);
}

// The FP32-flux / FP64-state form of curv_face_kernel (Rusanov and Roe).
template <int SCHEME, int FLUX>
__global__ void __launch_bounds__(128, 4) curv_face_f32_kernel(GridView g, StageView sv, int axis, double* fl) {
    if (sv.require_active && !sv.clock->active) return;
    constexpr int NST = SchemeInfo<SCHEME>::NST, CL = NST / 2 - 1;
    const int a = axis;
    int base[3], span[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const bool per = d < g.dim && g.bc_lo[d] == BC_PERIODIC;
        base[d] = d == a ? (per ? 0 : g.lo[d] - 1) : g.lo[d];
        span[d] = d == a ? (per ? g.n[d] : g.hi[d] - g.lo[d] + 1) : g.hi[d] - g.lo[d];
    }
    const long long total = (long long)span[0] * span[1] * span[2];
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    unsigned flags = 0, cut = 0, cores = 0;
    if (t < total) {
        int c[3];
        long long r = t;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            c[d] = base[d] + (int)(r % span[d]);
            r /= span[d];
        }
        const long long vs = g.vs;
        long long node[NST];
#pragma unroll
        for (int s = 0; s < NST; ++s) {
            int cc[3] = {c[0], c[1], c[2]};
            cc[a] = map_index(c[a] - CL + s, g.n[a], g.bc_lo[a], g.bc_hi[a]);
            node[s] = ((long long)cc[2] * g.n[1] + cc[1]) * g.n[0] + cc[0];
        }
        double qref[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) qref[v] = sv.qs[v * vs + node[CL]];
        float d[NST][5];
#pragma unroll
        for (int s = 0; s < NST; ++s)
#pragma unroll
            for (int v = 0; v < 5; ++v) d[s][v] = float(sv.qs[v * vs + node[s]] - qref[v]);
        const Ref32 ref = make_ref32(qref, g.gamma);
        const long long face = ((long long)c[2] * g.n[1] + c[1]) * g.n[0] + c[0];
        const double* gm = g.geom[a];
        const double n64[3] = {gm[face], gm[vs + face], gm[2 * vs + face]};
        const double area = gm[3 * vs + face];
        const float n[3] = {float(n64[0]), float(n64[1]), float(n64[2])};
        float F[5];
        curv_face_dev32<SCHEME, FLUX>(d, ref, n, float(g.gamma), F, flags, cut);
        if (SCHEME == TENO5) cores += 10;
        double fref[5];
        euler_flux_n(qref, n64, g.gamma, fref, flags);
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            const double x = (fref[v] + double(F[v])) * area;
            if (!isfinite(x)) flags |= FLAG_NONFINITE;
            fl[((long long)a * 5 + v) * vs + face] = x;
        }
    }
    flush_status(sv, flags, cores, cut);
}

// ---------------------------------------------------------------------------
// 2-D FP32-flux stage fused in one tile (the curvilinear form of
// tile2d_f32_body): the tile and its halo staged as FP32 deviations from the
// stage's reference node q_ref (ref_node, shared by every tile, so a
// tile-edge face has the same bits in both tiles); every x and y face of the
// tile from shared memory
// with its own normal and area, as the flux deviation dF * area; per node
// div = sum dF area (FP64) + (sum of the node's face cofactors) . F(q_ref),
// the second term in FP64 (on a curved grid the reference flux does not
// cancel between a node's faces).  No face fluxes round-trip through HBM.
// ---------------------------------------------------------------------------
template <int SCHEME, int FLUX, int TX, int TY>
__global__ void __launch_bounds__(TILE_THREADS, 3) curv_tile2d_f32_kernel(GridView g, StageView sv) {
    if (sv.require_active && !sv.clock->active) return;
    extern __shared__ float smem_c[];
    using S = TileShape<SCHEME, TX, TY>;
    constexpr int NST = S::NST, H = S::H, SX = S::SX, SY = S::SY, NFX = S::NFX, NFY = S::NFY;
    constexpr int NFXP = S::NFXP, NFYP = S::NFYP;
    const int ntx = (g.hi[0] - g.lo[0] + TX - 1) / TX;
    const int x0 = g.lo[0] + (blockIdx.x % ntx) * TX, y0 = g.lo[1] + (blockIdx.x / ntx) * TY;
    float* sq = smem_c;             // [5][SY][SX] deviations from qref
    float* fx = sq + 5 * SX * SY;   // [5][TY][TX+1]
    float* fy = fx + 5 * NFX;       // [5][TY+1][TX]
    const long long nx = g.n[0], vs = g.vs;
    unsigned flags = 0, cut = 0, cores = 0;
    double qref[5];
    load_ref(g, sv.qs, qref);
    const Ref32 ref = make_ref32(qref, g.gamma);
    for (int t = threadIdx.x; t < SX * SY; t += blockDim.x) {
        const int r = t / SX, c = t - r * SX;
        if ((r < H || r >= TY + H) && (c < H || c >= TX + H)) continue;
        const int gx = map_tile_index(x0 - H + c, g.n[0], g.bc_lo[0], g.bc_hi[0]);
        const int gy = map_tile_index(y0 - H + r, g.n[1], g.bc_lo[1], g.bc_hi[1]);
        const long long at = (long long)gy * nx + gx;
#pragma unroll
        for (int v = 0; v < 5; ++v) sq[v * SX * SY + t] = float(__ldg(sv.qs + v * vs + at) - qref[v]);
    }
    __syncthreads();
    const float gamma = float(g.gamma);
    // face (i | i+1) geometry sits at its lower node; only the periodic wrap
    // applies to that index
    auto lower = [&](int i, int a) { return i < 0 ? i + g.n[a] : i; };
    for (int f = threadIdx.x; f < NFXP + NFYP; f += blockDim.x) {
        float st[NST][5];
        float Ft[5];
        if (f < NFXP) {
            if (f >= NFX) continue;
            const int r = f / (TX + 1), c = f - r * (TX + 1);
            const int gy = y0 + r, gl = x0 - 1 + c;  // face between nodes gl and gl + 1 of row gy
            if (gy >= g.hi[1] || gl >= g.hi[0]) {
#pragma unroll
                for (int v = 0; v < 5; ++v) fx[v * NFX + f] = 0.f;
                continue;
            }
            const float* base = sq + (r + H) * SX + c;
#pragma unroll
            for (int s = 0; s < NST; ++s)
#pragma unroll
                for (int v = 0; v < 5; ++v) st[s][v] = base[v * SX * SY + s];
            const long long face = (long long)gy * nx + lower(gl, 0);
            const float n[3] = {float(g.geom[0][face]), float(g.geom[0][vs + face]), float(g.geom[0][2 * vs + face])};
            curv_face_dev32<SCHEME, FLUX>(st, ref, n, gamma, Ft, flags, cut);
            const float area = float(g.geom[0][3 * vs + face]);
#pragma unroll
            for (int v = 0; v < 5; ++v) fx[v * NFX + f] = Ft[v] * area;
        } else {
            const int k = f - NFXP;
            if (k >= NFY) continue;
            const int r = k / TX, c = k - r * TX;
            const int gx = x0 + c, gl = y0 - 1 + r;  // face between rows gl and gl + 1 of column gx
            if (gx >= g.hi[0] || gl >= g.hi[1]) {
#pragma unroll
                for (int v = 0; v < 5; ++v) fy[v * NFY + k] = 0.f;
                continue;
            }
            const float* base = sq + r * SX + (c + H);
#pragma unroll
            for (int s = 0; s < NST; ++s)
#pragma unroll
                for (int v = 0; v < 5; ++v) st[s][v] = base[v * SX * SY + s * SX];
            const long long face = (long long)lower(gl, 1) * nx + gx;
            const float n[3] = {float(g.geom[1][face]), float(g.geom[1][vs + face]), float(g.geom[1][2 * vs + face])};
            curv_face_dev32<SCHEME, FLUX>(st, ref, n, gamma, Ft, flags, cut);
            const float area = float(g.geom[1][3 * vs + face]);
#pragma unroll
            for (int v = 0; v < 5; ++v) fy[v * NFY + k] = Ft[v] * area;
        }
        if (SCHEME == TENO5) cores += 10;
    }
    __syncthreads();
    // physical flux tensor of q_ref (FP64): Fc = flux along axis c
    double Fc[3][5];
    {
        const double rho = qref[0];
        const double u[3] = {qref[1] / rho, qref[2] / rho, qref[3] / rho};
        const double p = (g.gamma - 1.0) * (qref[4] - 0.5 * (qref[1] * u[0] + qref[2] * u[1] + qref[3] * u[2]));
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            Fc[c][0] = qref[1 + c];
#pragma unroll
            for (int k = 0; k < 3; ++k) Fc[c][1 + k] = qref[1 + k] * u[c] + (k == c ? p : 0.0);
            Fc[c][4] = (qref[4] + p) * u[c];
        }
    }
    const double dt = sv.clock->dt;
    double sr = 0.0;
    for (int nd = threadIdx.x; nd < TX * TY; nd += blockDim.x) {
        const int r = nd / TX, c = nd - r * TX;
        const int gx = x0 + c, gy = y0 + r;
        if (gx >= g.hi[0] || gy >= g.hi[1]) continue;
        const long long node = (long long)gy * nx + gx;
        // the node's net face cofactor: upper minus lower face of each axis
        const long long fxl = (long long)gy * nx + lower(gx - 1, 0), fyl = (long long)lower(gy - 1, 1) * nx + gx;
        double gc[3];
#pragma unroll
        for (int k = 0; k < 3; ++k)
            gc[k] = g.geom[0][k * vs + node] * g.geom[0][3 * vs + node] - g.geom[0][k * vs + fxl] * g.geom[0][3 * vs + fxl] +
                    g.geom[1][k * vs + node] * g.geom[1][3 * vs + node] - g.geom[1][k * vs + fyl] * g.geom[1][3 * vs + fyl];
        double div[5], qn[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            const float* fxv = fx + v * NFX + r * (TX + 1) + c;
            const float* fyv = fy + v * NFY + r * TX + c;
            // FP32 face deviations with exact FP64 differences, the reference
            // flux term in FP64
            div[v] = (double(fxv[1]) - double(fxv[0])) + (double(fyv[TX]) - double(fyv[0])) +
                     (gc[0] * Fc[0][v] + gc[1] * Fc[1][v] + gc[2] * Fc[2][v]);
            qn[v] = __ldg(sv.qs + v * vs + node);
        }
        finish_node_j<true>(g, sv, dt, node, qn, div, g.node_jac[node], flags, sr);
    }
    flush_status(sv, flags, cores, cut);
    if (sv.mode & MODE_CFL) flush_cfl_block(g, sv.clock, sr);
}

// The FP64 form of the fused 2-D tile: the state staged as is, full face
// fluxes (times the area) in shared memory, div = dFx + dFy per node.
template <int SCHEME, int FLUX, int TX, int TY>
__global__ void __launch_bounds__(TILE_THREADS, 2) curv_tile2d_kernel(GridView g, StageView sv) {
    if (sv.require_active && !sv.clock->active) return;
    extern __shared__ double smem_d[];
    using S = TileShape<SCHEME, TX, TY>;
    constexpr int NST = S::NST, W = S::NST == 8 ? 7 : (S::NST == 4 ? 4 : 5), H = S::H, SX = S::SX, SY = S::SY;
    constexpr int NFX = S::NFX, NFY = S::NFY, NFXP = S::NFXP, NFYP = S::NFYP;
    const int ntx = (g.hi[0] - g.lo[0] + TX - 1) / TX;
    const int x0 = g.lo[0] + (blockIdx.x % ntx) * TX, y0 = g.lo[1] + (blockIdx.x / ntx) * TY;
    double* sq = smem_d;            // [5][SY][SX]
    double* fx = sq + 5 * SX * SY;  // [5][TY][TX+1]
    double* fy = fx + 5 * NFX;      // [5][TY+1][TX]
    const long long nx = g.n[0], vs = g.vs;
    unsigned flags = 0, cut = 0, cores = 0;
    for (int t = threadIdx.x; t < SX * SY; t += blockDim.x) {
        const int r = t / SX, c = t - r * SX;
        if ((r < H || r >= TY + H) && (c < H || c >= TX + H)) continue;
        const int gx = map_tile_index(x0 - H + c, g.n[0], g.bc_lo[0], g.bc_hi[0]);
        const int gy = map_tile_index(y0 - H + r, g.n[1], g.bc_lo[1], g.bc_hi[1]);
        const long long at = (long long)gy * nx + gx;
#pragma unroll
        for (int v = 0; v < 5; ++v) sq[v * SX * SY + t] = __ldg(sv.qs + v * vs + at);
    }
    __syncthreads();
    auto lower = [&](int i, int a) { return i < 0 ? i + g.n[a] : i; };
    for (int f = threadIdx.x; f < NFXP + NFYP; f += blockDim.x) {
        double st[NST][5];
        const double* gm;
        double* out;
        long long face;
        int slot, stride;
        const double* base;
        if (f < NFXP) {
            if (f >= NFX) continue;
            const int r = f / (TX + 1), c = f - r * (TX + 1);
            const int gy = y0 + r, gl = x0 - 1 + c;
            if (gy >= g.hi[1] || gl >= g.hi[0]) {
#pragma unroll
                for (int v = 0; v < 5; ++v) fx[v * NFX + f] = 0.0;
                continue;
            }
            base = sq + (r + H) * SX + c;
            stride = 1;
            gm = g.geom[0];
            face = (long long)gy * nx + lower(gl, 0);
            out = fx;
            slot = f;
        } else {
            const int k = f - NFXP;
            if (k >= NFY) continue;
            const int r = k / TX, c = k - r * TX;
            const int gx = x0 + c, gl = y0 - 1 + r;
            if (gx >= g.hi[0] || gl >= g.hi[1]) {
#pragma unroll
                for (int v = 0; v < 5; ++v) fy[v * NFY + k] = 0.0;
                continue;
            }
            base = sq + r * SX + (c + H);
            stride = SX;
            gm = g.geom[1];
            face = (long long)lower(gl, 1) * nx + gx;
            out = fy;
            slot = k;
        }
#pragma unroll
        for (int s2 = 0; s2 < NST; ++s2)
#pragma unroll
            for (int v = 0; v < 5; ++v) st[s2][v] = base[v * SX * SY + s2 * stride];
        const double n[3] = {gm[face], gm[vs + face], gm[2 * vs + face]};
        const double area = gm[3 * vs + face];
        double qavg[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) qavg[v] = 0.5 * (st[NST / 2 - 1][v] + st[NST / 2][v]);
        CharBasis e;
        char_basis_n(qavg, n, g.gamma, e, flags);
        double qL[5] = {0.0, 0.0, 0.0, 0.0, 0.0}, qR[5] = {0.0, 0.0, 0.0, 0.0, 0.0}, F[5];
        recon_field<0, SCHEME, NST, W, double>(e, st, qL, qR, flags, cut);
        recon_field<1, SCHEME, NST, W, double>(e, st, qL, qR, flags, cut);
        recon_field<2, SCHEME, NST, W, double>(e, st, qL, qR, flags, cut);
        recon_field<3, SCHEME, NST, W, double>(e, st, qL, qR, flags, cut);
        recon_field<4, SCHEME, NST, W, double>(e, st, qL, qR, flags, cut);
        flux_n<FLUX>(qL, qR, n, g.gamma, F, flags);
        const int nf = out == fx ? NFX : NFY;
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            const double x = F[v] * area;
            if (!isfinite(x)) flags |= FLAG_NONFINITE;
            out[v * nf + slot] = x;
        }
        if (SCHEME == TENO5) cores += 10;
    }
    __syncthreads();
    const double dt = sv.clock->dt;
    double sr = 0.0;
    for (int nd = threadIdx.x; nd < TX * TY; nd += blockDim.x) {
        const int r = nd / TX, c = nd - r * TX;
        const int gx = x0 + c, gy = y0 + r;
        if (gx >= g.hi[0] || gy >= g.hi[1]) continue;
        const long long node = (long long)gy * nx + gx;
        double div[5], qn[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            const double* fxv = fx + v * NFX + r * (TX + 1) + c;
            const double* fyv = fy + v * NFY + r * TX + c;
            div[v] = 0.0;
            div[v] += fxv[1] - fxv[0];
            div[v] += fyv[TX] - fyv[0];
            qn[v] = sq[v * SX * SY + (r + H) * SX + (c + H)];
        }
        finish_node_j<true>(g, sv, dt, node, qn, div, g.node_jac[node], flags, sr);
    }
    flush_status(sv, flags, cores, cut);
    if (sv.mode & MODE_CFL) flush_cfl_block(g, sv.clock, sr);
}

// Divergence and stage update of the solved nodes.
__global__ void __launch_bounds__(256) curv_stage_kernel(GridView g, StageView sv, const double* __restrict__ fl) {
    if (sv.require_active && !sv.clock->active) return;
    const long long cx = g.hi[0] - g.lo[0], cy = g.hi[1] - g.lo[1], cz = g.hi[2] - g.lo[2];
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    unsigned flags = 0;
    double sr = 0.0;
    if (t < cx * cy * cz) {
        const int c[3] = {g.lo[0] + (int)(t % cx), g.lo[1] + (int)((t / cx) % cy), g.lo[2] + (int)(t / (cx * cy))};
        const long long vs = g.vs;
        const long long node = ((long long)c[2] * g.n[1] + c[1]) * g.n[0] + c[0];
        double div[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        for (int d = 0; d < g.dim; ++d) {
            // the lower face is stored at node i - 1 (a face index, not a
            // value read: only the periodic wrap applies)
            int cl[3] = {c[0], c[1], c[2]};
            cl[d] = c[d] - 1 < 0 ? c[d] - 1 + g.n[d] : c[d] - 1;
            const long long lower = ((long long)cl[2] * g.n[1] + cl[1]) * g.n[0] + cl[0];
#pragma unroll
            for (int v = 0; v < 5; ++v)
                div[v] += fl[((long long)d * 5 + v) * vs + node] - fl[((long long)d * 5 + v) * vs + lower];
        }
        double qn[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) qn[v] = sv.qs[v * vs + node];
        finish_node_j<true>(g, sv, sv.clock->dt, node, qn, div, g.node_jac[node], flags, sr);
    }
    if (flags) atomicOr(sv.flags, flags);
    if (sv.mode & MODE_CFL) flush_cfl_block(g, sv.clock, sr);
}

// ---------------------------------------------------------------------------
cudaError_t launch_curv_geometry(const GridView& g, const double* nm, double* const geom[3], unsigned* flags,
                                 cudaStream_t st) {
    const long long nodes = (long long)g.n[0] * g.n[1] * g.n[2];
    const unsigned blocks = (unsigned)std::min<long long>((nodes + 255) / 256, 148LL * 16);
    curv_geometry_kernel<<<blocks, 256, 0, st>>>(g, nm, geom[0], geom[1], geom[2], flags);
    return cudaGetLastError();
}

template <int SCHEME, int FLUX>
static cudaError_t launch_curv_faces(const GridView& g, const StageView& sv, int axis, double* fl, cudaStream_t st) {
    long long total = 1;
    for (int d = 0; d < 3; ++d) {
        const bool per = d < g.dim && g.bc_lo[d] == BC_PERIODIC;
        total *= d == axis ? (per ? g.n[d] : g.hi[d] - g.lo[d] + 1) : g.hi[d] - g.lo[d];
    }
    curv_face_kernel<SCHEME, FLUX><<<(unsigned)((total + 127) / 128), 128, 0, st>>>(g, sv, axis, fl);
    return cudaGetLastError();
}

template <int SCHEME, int FLUX>
static cudaError_t launch_curv_faces32(const GridView& g, const StageView& sv, int axis, double* fl, cudaStream_t st) {
    long long total = 1;
    for (int d = 0; d < 3; ++d) {
        const bool per = d < g.dim && g.bc_lo[d] == BC_PERIODIC;
        total *= d == axis ? (per ? g.n[d] : g.hi[d] - g.lo[d] + 1) : g.hi[d] - g.lo[d];
    }
    curv_face_f32_kernel<SCHEME, FLUX><<<(unsigned)((total + 127) / 128), 128, 0, st>>>(g, sv, axis, fl);
    return cudaGetLastError();
}

template <int SCHEME>
static cudaError_t launch_curv_faces_f(int flux, int prec64, const GridView& g, const StageView& sv, int axis,
                                       double* fl, cudaStream_t st) {
    if (!prec64) {
        if (flux == RUSANOV) return launch_curv_faces32<SCHEME, RUSANOV>(g, sv, axis, fl, st);
        if (flux == ROE) return launch_curv_faces32<SCHEME, ROE>(g, sv, axis, fl, st);
        return cudaErrorInvalidValue;
    }
    switch (flux) {
    case RUSANOV: return launch_curv_faces<SCHEME, RUSANOV>(g, sv, axis, fl, st);
    case ROE: return launch_curv_faces<SCHEME, ROE>(g, sv, axis, fl, st);
    case STEGER: return launch_curv_faces<SCHEME, STEGER>(g, sv, axis, fl, st);
    case LAXF: return launch_curv_faces<SCHEME, LAXF>(g, sv, axis, fl, st);
    }
    return cudaErrorInvalidValue;
}

template <int SCHEME, int FLUX>
static cudaError_t launch_curv_tile2d(const GridView& g, const StageView& sv, cudaStream_t st) {
    constexpr int TX = 22, TY = 22;
    using S = TileShape<SCHEME, TX, TY>;
    const int ntx = (g.hi[0] - g.lo[0] + TX - 1) / TX, nty = (g.hi[1] - g.lo[1] + TY - 1) / TY;
    const size_t smem = sizeof(float) * S::ELEMS;
    auto kern = curv_tile2d_f32_kernel<SCHEME, FLUX, TX, TY>;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    kern<<<ntx * nty, TILE_THREADS, smem, st>>>(g, sv);
    return cudaGetLastError();
}

template <int SCHEME, int FLUX>
static cudaError_t launch_curv_tile2d64(const GridView& g, const StageView& sv, cudaStream_t st) {
    constexpr int TX = 22, TY = 22;
    using S = TileShape<SCHEME, TX, TY>;
    const int ntx = (g.hi[0] - g.lo[0] + TX - 1) / TX, nty = (g.hi[1] - g.lo[1] + TY - 1) / TY;
    const size_t smem = sizeof(double) * S::ELEMS;
    auto kern = curv_tile2d_kernel<SCHEME, FLUX, TX, TY>;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    kern<<<ntx * nty, TILE_THREADS, smem, st>>>(g, sv);
    return cudaGetLastError();
}

template <int SCHEME>
static cudaError_t launch_curv_tile2d_f(int flux, int prec64, const GridView& g, const StageView& sv,
                                        cudaStream_t st) {
    if (prec64) {
        switch (flux) {
        case RUSANOV: return launch_curv_tile2d64<SCHEME, RUSANOV>(g, sv, st);
        case ROE: return launch_curv_tile2d64<SCHEME, ROE>(g, sv, st);
        case STEGER: return launch_curv_tile2d64<SCHEME, STEGER>(g, sv, st);
        case LAXF: return launch_curv_tile2d64<SCHEME, LAXF>(g, sv, st);
        }
        return cudaErrorInvalidValue;
    }
    if (flux == RUSANOV) return launch_curv_tile2d<SCHEME, RUSANOV>(g, sv, st);
    if (flux == ROE) return launch_curv_tile2d<SCHEME, ROE>(g, sv, st);
    return cudaErrorInvalidValue;
}

// One stage on a curvilinear grid: the face fluxes of every active axis, then
// the divergence and stage update (sv.mode: MODE_FINAL with optional
// MODE_RESIDUAL / MODE_CFL); 2-D FP32-flux grids run the fused tile kernel.
cudaError_t launch_curv_stage(int scheme, int flux, int prec64, int tiles, const GridView& g, const StageView& sv,
                              double* fl, cudaStream_t st) {
    if (g.dim == 2 && tiles) {
        switch (scheme) {
        case WENO5: return launch_curv_tile2d_f<WENO5>(flux, prec64, g, sv, st);
        case TENO5: return launch_curv_tile2d_f<TENO5>(flux, prec64, g, sv, st);
        case WENO3: return launch_curv_tile2d_f<WENO3>(flux, prec64, g, sv, st);
        case WENO7: return launch_curv_tile2d_f<WENO7>(flux, prec64, g, sv, st);
        default: return cudaErrorInvalidValue;
        }
    }
    for (int axis = 0; axis < g.dim; ++axis) {
        cudaError_t e;
        switch (scheme) {
        case WENO5: e = launch_curv_faces_f<WENO5>(flux, prec64, g, sv, axis, fl, st); break;
        case TENO5: e = launch_curv_faces_f<TENO5>(flux, prec64, g, sv, axis, fl, st); break;
        case WENO3: e = launch_curv_faces_f<WENO3>(flux, prec64, g, sv, axis, fl, st); break;
        case WENO7: e = launch_curv_faces_f<WENO7>(flux, prec64, g, sv, axis, fl, st); break;
        default: return cudaErrorInvalidValue;
        }
        if (e != cudaSuccess) return e;
    }
    const long long solved = (long long)(g.hi[0] - g.lo[0]) * (g.hi[1] - g.lo[1]) * (g.hi[2] - g.lo[2]);
    curv_stage_kernel<<<(unsigned)((solved + 255) / 256), 256, 0, st>>>(g, sv, fl);
    return cudaGetLastError();
}

}  // namespace sfg
