/*
 * sf_oracle.c -- CPU oracle for the density-based explicit Euler path.
 *
 * TEST INFRASTRUCTURE ONLY (see sf_oracle.h).  A plain-C restatement of the
 * reference algorithm, written to keep the reference's order of floating-point
 * operations so that, built with the same flags, it agrees bit for bit with
 * the reference translation units compiled under oracle/_ref.
 *
 * Reference files cited below are paths inside the sonicSolver source tree.
 */
#include "sf_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define NV 5

/* ------------------------------------------------------------------ */
/* Scalar reconstruction cores                                         */
/* ------------------------------------------------------------------ */

static int all_finite(const double* v, int n) {
    for (int s = 0; s < n; ++s)
        if (!isfinite(v[s])) return 0;
    return 1;
}

/* WENO3-JS, SF_WENO3.cpp:42-57 (eps 1e-6, d = 1/3, 2/3). */
double sfo_weno3_core(const double* v) {
    double p0 = (-v[0] + 5.0 * v[1] + 2.0 * v[2]) / 6.0;
    double p1 = (2.0 * v[1] + 5.0 * v[2] - v[3]) / 6.0;
    const double d0 = 1.0 / 3.0, d1 = 2.0 / 3.0;
    double b0 = (v[2] - v[0]) * (v[2] - v[0]);
    double b1 = (v[3] - v[1]) * (v[3] - v[1]);
    const double eps = 1e-6;
    double a0 = d0 / ((eps + b0) * (eps + b0));
    double a1 = d1 / ((eps + b1) * (eps + b1));
    double sumA = a0 + a1;
    if (!isfinite(sumA) || sumA <= 0.0) return NAN;
    return (a0 * p0 + a1 * p1) / sumA;
}

static double sq(double x) { return x * x; }  /* std::pow(x, 2) is exact x*x */

/* WENO5-JS, SF_WENO5.cpp:42-62 (eps 1e-6, power 2, d = 0.1, 0.6, 0.3). */
double sfo_weno5_core(const double* v) {
    double p0 = (2.0 * v[0] - 7.0 * v[1] + 11.0 * v[2]) / 6.0;
    double p1 = (-1.0 * v[1] + 5.0 * v[2] + 2.0 * v[3]) / 6.0;
    double p2 = (2.0 * v[2] + 5.0 * v[3] - 1.0 * v[4]) / 6.0;
    const double d0 = 0.1, d1 = 0.6, d2 = 0.3;
    double b0 = 13.0 / 12.0 * sq(v[0] - 2.0 * v[1] + v[2]) + 0.25 * sq(v[0] - 4.0 * v[1] + 3.0 * v[2]);
    double b1 = 13.0 / 12.0 * sq(v[1] - 2.0 * v[2] + v[3]) + 0.25 * sq(v[1] - v[3]);
    double b2 = 13.0 / 12.0 * sq(v[2] - 2.0 * v[3] + v[4]) + 0.25 * sq(3.0 * v[2] - 4.0 * v[3] + v[4]);
    const double eps = 1e-6;
    double a0 = d0 / sq(eps + b0);
    double a1 = d1 / sq(eps + b1);
    double a2 = d2 / sq(eps + b2);
    double sumA = a0 + a1 + a2;
    if (!isfinite(sumA) || sumA <= 0.0) return NAN;
    return (a0 * p0 + a1 * p1 + a2 * p2) / sumA;
}

/* TENO5, SF_TENO5.cpp:44-92 (C = 1, q = 6, eps = 1e-40, CT = 1e-5).
 * cut_mask bit k is set when sub-stencil k is cut off.  Returns NAN when all
 * three are cut (the reference exits the process there). */
double sfo_teno5_core(const double* v, int* cut_mask) {
    const double p0 = (2.0 * v[0] - 7.0 * v[1] + 11.0 * v[2]) / 6.0;
    const double p1 = (-1.0 * v[1] + 5.0 * v[2] + 2.0 * v[3]) / 6.0;
    const double p2 = (2.0 * v[2] + 5.0 * v[3] - 1.0 * v[4]) / 6.0;
    const double b0 = 13.0 / 12.0 * sq(v[0] - 2.0 * v[1] + v[2]) + 0.25 * sq(v[0] - 4.0 * v[1] + 3.0 * v[2]);
    const double b1 = 13.0 / 12.0 * sq(v[1] - 2.0 * v[2] + v[3]) + 0.25 * sq(v[1] - v[3]);
    const double b2 = 13.0 / 12.0 * sq(v[2] - 2.0 * v[3] + v[4]) + 0.25 * sq(3.0 * v[2] - 4.0 * v[3] + v[4]);
    const double d0 = 0.1, d1 = 0.6, d2 = 0.3;
    const double eps = 1.0e-40, ct = 1.0e-5;
    const double tau5 = fabs(b0 - b2);
    const double g0 = pow(1.0 + tau5 / (b0 + eps), 6);
    const double g1 = pow(1.0 + tau5 / (b1 + eps), 6);
    const double g2 = pow(1.0 + tau5 / (b2 + eps), 6);
    const double gsum = g0 + g1 + g2;
    if (!isfinite(gsum) || gsum <= 0.0) return NAN;
    const double c0 = (g0 / gsum < ct) ? 0.0 : 1.0;
    const double c1 = (g1 / gsum < ct) ? 0.0 : 1.0;
    const double c2 = (g2 / gsum < ct) ? 0.0 : 1.0;
    if (cut_mask) *cut_mask = (c0 == 0.0) | ((c1 == 0.0) << 1) | ((c2 == 0.0) << 2);
    const double active = d0 * c0 + d1 * c1 + d2 * c2;
    if (active <= 0.0) return NAN;
    return (d0 * c0 * p0 + d1 * c1 * p1 + d2 * c2 * p2) / active;
}

/* 4-point smoothness indicator of WENO7, SF_WENO7.cpp:41-69: the integral
 * over [a, b] of the squared derivatives of the cubic through v. */
static double beta4(const double v[4], double a, double b) {
    double d1 = v[1] - v[0];
    double d2 = (v[2] - 2.0 * v[1] + v[0]) * 0.5;
    double d3 = (v[3] - 3.0 * v[2] + 3.0 * v[1] - v[0]) / 6.0;
    double A = d1 - d2 + 2.0 * d3;
    double B = 2.0 * d2 - 6.0 * d3;
    double C = 3.0 * d3;
    double i1 = b - a;
    double i2 = b * b - a * a;
    double i3 = b * b * b / 3.0 - a * a * a / 3.0;
    double b2a = b * b, a2a = a * a;
    double i4 = b2a * b2a / 2.0 - a2a * a2a / 2.0;
    double i5 = b * b * b * b * b / 5.0 - a * a * a * a * a / 5.0;
    double beta1 = A * A * i1 + A * B * i2 + (B * B + 2.0 * A * C) * i3 + B * C * i4 + C * C * i5;
    double D = 2.0 * d2 - 6.0 * d3;
    double E = 6.0 * d3;
    double beta2 = D * D * i1 + D * E * i2 + E * E * i3;
    double beta3 = 36.0 * d3 * d3 * i1;
    return beta1 + beta2 + beta3;
}

/* WENO7-JS, SF_WENO7.cpp:71-98. */
double sfo_weno7_core(const double* v) {
    double p0 = (-3.0 * v[0] + 13.0 * v[1] - 23.0 * v[2] + 25.0 * v[3]) / 12.0;
    double p1 = (v[1] - 5.0 * v[2] + 13.0 * v[3] + 3.0 * v[4]) / 12.0;
    double p2 = (-v[2] + 7.0 * v[3] + 7.0 * v[4] - v[5]) / 12.0;
    double p3 = (3.0 * v[3] + 13.0 * v[4] - 5.0 * v[5] + v[6]) / 12.0;
    const double d0 = 1.0 / 35.0, d1 = 12.0 / 35.0, d2 = 18.0 / 35.0, d3 = 4.0 / 35.0;
    double s0[4] = {v[0], v[1], v[2], v[3]};
    double s1[4] = {v[1], v[2], v[3], v[4]};
    double s2[4] = {v[2], v[3], v[4], v[5]};
    double s3[4] = {v[3], v[4], v[5], v[6]};
    double b0 = beta4(s0, 2.5, 3.5);
    double b1 = beta4(s1, 1.5, 2.5);
    double b2 = beta4(s2, 0.5, 1.5);
    double b3 = beta4(s3, -0.5, 0.5);
    const double eps = 1e-6;
    double a0 = d0 / ((eps + b0) * (eps + b0));
    double a1 = d1 / ((eps + b1) * (eps + b1));
    double a2 = d2 / ((eps + b2) * (eps + b2));
    double a3 = d3 / ((eps + b3) * (eps + b3));
    double sumA = a0 + a1 + a2 + a3;
    if (!isfinite(sumA) || sumA <= 0.0) return NAN;
    return (a0 * p0 + a1 * p1 + a2 * p2 + a3 * p3) / sumA;
}

/* ------------------------------------------------------------------ */
/* Thermodynamics and eigen-structure                                  */
/* ------------------------------------------------------------------ */

/* requirePhysicalState, SF_utility.h:24-29,46-66: p from conserved state. */
static int physical_pressure(const double* q, double gamma, double* p) {
    if (!isfinite(q[0]) || !isfinite(q[1]) || !isfinite(q[2]) || !isfinite(q[3]) ||
        !isfinite(q[4]))
        return SFO_ERR_NONFINITE;
    if (q[0] <= 0.0) return SFO_ERR_STATE;
    double invRho = 1.0 / q[0];
    double ke = 0.5 * (q[1] * q[1] + q[2] * q[2] + q[3] * q[3]) * invRho;
    double pr = (gamma - 1.0) * (q[4] - ke);
    if (!isfinite(pr)) return SFO_ERR_NONFINITE;
    if (pr <= 0.0) return SFO_ERR_STATE;
    *p = pr;
    return SFO_OK;
}

/* Riemann::buildCharacteristicMatrix, SF_riemann.cpp:69-123. */
int sfo_char_matrix(const double* q, const double* n, double gamma, double* L, double* R) {
    double p;
    int err = physical_pressure(q, gamma, &p);
    if (err) return err;
    double r = q[0];
    double invR = 1.0 / r;
    double u = q[1] * invR, v = q[2] * invR, w = q[3] * invR;
    double e = q[4];
    double q2 = u * u + v * v + w * w;
    double c = sqrt(gamma * p * invR);
    double H = (e + p) * invR;
    double n1 = n[0], n2 = n[1], n3 = n[2];
    double l1, l2, l3, m1, m2, m3;
    if (fabs(n3) <= fabs(n2)) {
        double ss = sqrt(n1 * n1 + n2 * n2);
        l1 = -n2 / ss; l2 = n1 / ss; l3 = 0.0;
    } else {
        double ss = sqrt(n1 * n1 + n3 * n3);
        l1 = -n3 / ss; l2 = 0.0; l3 = n1 / ss;
    }
    m1 = n2 * l3 - n3 * l2;
    m2 = n3 * l1 - n1 * l3;
    m3 = n1 * l2 - n2 * l1;
    double un = u * n1 + v * n2 + w * n3;
    double ul = u * l1 + v * l2 + w * l3;
    double um = u * m1 + v * m2 + w * m3;
    double b1 = (gamma - 1.0) / (c * c);
    double b2 = 0.5 * b1;
    double x1 = 1.0 / (2.0 * c);
    double Lm[25] = {
        1.0 - b2 * q2, b1 * u, b1 * v, b1 * w, -b1,
        -ul, l1, l2, l3, 0.0,
        -um, m1, m2, m3, 0.0,
        0.5 * b2 * q2 + x1 * un, -x1 * n1 - b2 * u, -x1 * n2 - b2 * v, -x1 * n3 - b2 * w, b2,
        0.5 * b2 * q2 - x1 * un, x1 * n1 - b2 * u, x1 * n2 - b2 * v, x1 * n3 - b2 * w, b2};
    double Rm[25] = {
        1.0, 0.0, 0.0, 1.0, 1.0,
        u, l1, m1, u - c * n1, u + c * n1,
        v, l2, m2, v - c * n2, v + c * n2,
        w, l3, m3, w - c * n3, w + c * n3,
        0.5 * q2, ul, um, H - c * un, H + c * un};
    memcpy(L, Lm, sizeof Lm);
    memcpy(R, Rm, sizeof Rm);
    return SFO_OK;
}

/* Riemann::gemv5, SF_riemann.h:33-37. */
static void gemv5(const double* M, const double* V, double* out) {
    for (int i = 0; i < 5; ++i)
        out[i] = M[i * 5 + 0] * V[0] + M[i * 5 + 1] * V[1] + M[i * 5 + 2] * V[2] +
                 M[i * 5 + 3] * V[3] + M[i * 5 + 4] * V[4];
}

typedef struct { double vel[3]; double p; double c; } closed_state;

/* SingleFluidStateModel::close + PerfectGasEOS::fromDensityEnergy
 * (SF_singleFluidStateModel.cpp:49-73, SF_perfectGasEOS.h:26-33). */
static int close_state(const double* q, double gamma, closed_state* s) {
    if (!all_finite(q, 5)) return SFO_ERR_NONFINITE;
    const double rho = q[0];
    if (rho <= 0.0) return SFO_ERR_STATE;
    for (int d = 0; d < 3; ++d) s->vel[d] = q[1 + d] / rho;
    const double kinetic = 0.5 * rho * (s->vel[0] * s->vel[0] + s->vel[1] * s->vel[1] + s->vel[2] * s->vel[2]);
    const double eint = q[4] - kinetic;
    const double e = eint / rho;
    const double thermal = e - 0.0;
    const double p = (gamma - 1.0) * rho * thermal;
    if (!isfinite(p)) return SFO_ERR_NONFINITE;
    if (p <= 0.0) return SFO_ERR_STATE;
    s->p = p;
    s->c = sqrt(gamma * p / rho);
    return SFO_OK;
}

/* RusanovEOS::faceFlux, SF_rusanovEOS.cpp:14-32,47-77. */
int sfo_rusanov_flux(const double* qL, const double* qR, const double* n, double gamma, double* out) {
    closed_state l, r;
    int err = close_state(qL, gamma, &l);
    if (err) return err;
    err = close_state(qR, gamma, &r);
    if (err) return err;
    const double unL = l.vel[0] * n[0] + l.vel[1] * n[1] + l.vel[2] * n[2];
    const double unR = r.vel[0] * n[0] + r.vel[1] * n[1] + r.vel[2] * n[2];
    double fL[5], fR[5];
    fL[0] = qL[0] * unL;
    fR[0] = qR[0] * unR;
    for (int d = 0; d < 3; ++d) {
        fL[1 + d] = qL[1 + d] * unL + l.p * n[d];
        fR[1 + d] = qR[1 + d] * unR + r.p * n[d];
    }
    fL[4] = (qL[4] + l.p) * unL;
    fR[4] = (qR[4] + r.p) * unR;
    const double aL = fabs(unL) + l.c, aR = fabs(unR) + r.c;
    const double lambda = aL < aR ? aR : aL;   /* std::max(aL, aR) */
    if (!isfinite(lambda) || lambda <= 0.0) return SFO_ERR_NONFINITE;
    for (int v = 0; v < 5; ++v)
        out[v] = 0.5 * (fL[v] + fR[v]) - 0.5 * lambda * (qR[v] - qL[v]);
    return SFO_OK;
}

/* physicalEulerFlux, SF_face.h:112-127. */
static int physical_euler_flux(const double* q, const double* n, double gamma, double* f) {
    const double rho = q[0];
    const double u = q[1] / rho, v = q[2] / rho, w = q[3] / rho;
    double p;
    int err = physical_pressure(q, gamma, &p);
    if (err) return err;
    const double un = u * n[0] + v * n[1] + w * n[2];
    f[0] = rho * un;
    f[1] = rho * u * un + p * n[0];
    f[2] = rho * v * un + p * n[1];
    f[3] = rho * w * un + p * n[2];
    f[4] = (q[4] + p) * un;
    return SFO_OK;
}

/* RoeFlux::flux with Harten entropy fix (delta = 0.1 a), SF_roe.cpp:20-111. */
int sfo_roe_flux(const double* qL, const double* qR, const double* n, double gamma, double* out) {
    const double gm1 = gamma - 1.0;
    double pL, pR;
    int err = physical_pressure(qL, gamma, &pL);
    if (err) return err;
    err = physical_pressure(qR, gamma, &pR);
    if (err) return err;
    const double invRL = 1.0 / qL[0];
    const double uL = qL[1] * invRL, vL = qL[2] * invRL, wL = qL[3] * invRL;
    const double hL = (qL[4] + pL) * invRL;
    const double invRR = 1.0 / qR[0];
    const double uR = qR[1] * invRR, vR = qR[2] * invRR, wR = qR[3] * invRR;
    const double hR = (qR[4] + pR) * invRR;
    const double sL = sqrt(qL[0]), sR = sqrt(qR[0]);
    const double ss = sL + sR;
    const double uRoe = (sL * uL + sR * uR) / ss;
    const double vRoe = (sL * vL + sR * vR) / ss;
    const double wRoe = (sL * wL + sR * wR) / ss;
    const double hRoe = (sL * hL + sR * hR) / ss;
    const double q2Roe = uRoe * uRoe + vRoe * vRoe + wRoe * wRoe;
    const double a2Roe = gm1 * (hRoe - 0.5 * q2Roe);
    if (!isfinite(a2Roe) || a2Roe <= 0.0) return SFO_ERR_ROE_SOUND;
    const double aRoe = sqrt(a2Roe);
    const double unRoe = uRoe * n[0] + vRoe * n[1] + wRoe * n[2];
    const double lambda[5] = {unRoe, unRoe, unRoe, unRoe + aRoe, unRoe - aRoe};
    double absLambda[5];
    const double entropyEps = 0.1 * aRoe;
    for (int m = 0; m < 5; ++m) {
        const double value = fabs(lambda[m]);
        if (value < 2.0 * entropyEps)
            absLambda[m] = 0.5 * (value * value / (2.0 * entropyEps) + entropyEps);
        else
            absLambda[m] = value;
    }
    double dQ[5];
    for (int v = 0; v < 5; ++v) dQ[v] = qR[v] - qL[v];
    const double rhoRoe = sL * sR;
    double qRoe[5];
    qRoe[0] = rhoRoe;
    qRoe[1] = rhoRoe * uRoe;
    qRoe[2] = rhoRoe * vRoe;
    qRoe[3] = rhoRoe * wRoe;
    qRoe[4] = rhoRoe * (0.5 * q2Roe + a2Roe / gm1);
    double Lm[25], Rm[25];
    err = sfo_char_matrix(qRoe, n, gamma, Lm, Rm);
    if (err) return err;
    double alpha[5];
    gemv5(Lm, dQ, alpha);
    double diss[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (int wave = 0; wave < 5; ++wave) {
        const double strength = absLambda[wave] * alpha[wave];
        for (int v = 0; v < 5; ++v) diss[v] += Rm[v * 5 + wave] * strength;
    }
    double fL[5], fR[5];
    err = physical_euler_flux(qL, n, gamma, fL);
    if (err) return err;
    err = physical_euler_flux(qR, n, gamma, fR);
    if (err) return err;
    for (int v = 0; v < 5; ++v) out[v] = 0.5 * (fL[v] + fR[v] - diss[v]);
    return SFO_OK;
}

/* ------------------------------------------------------------------ */
/* Characteristic face flux                                            */
/* Riemann::splitStegerWarming, SF_riemann.cpp:15-67: F+ and F- of one state
 * with the entropy-fixed eigenvalue split (eps = 0.01). */
static int steger_split(const double* Q, const double* n, double gamma, double* fpos, double* fneg) {
    const double r = Q[0];
    double p;
    int err = physical_pressure(Q, gamma, &p);
    if (err) return err;
    const double invR = 1.0 / r;
    const double u = Q[1] * invR, v = Q[2] * invR, w = Q[3] * invR;
    const double q2 = u * u + v * v + w * w;
    const double a = sqrt(gamma * p * invR);
    const double un = u * n[0] + v * n[1] + w * n[2];
    const double lam[5] = {un, un, un, un + a, un - a};
    double lp[5], lm[5];
    const double eps_sw = 0.01;
    for (int i = 0; i < 5; ++i) {
        if (fabs(lam[i]) < 2.0 * eps_sw) {
            lp[i] = 0.5 * (lam[i] * lam[i] / (4.0 * eps_sw) + lam[i] + eps_sw);
            lm[i] = lam[i] - lp[i];
        } else {
            lp[i] = 0.5 * (lam[i] + fabs(lam[i]));
            lm[i] = 0.5 * (lam[i] - fabs(lam[i]));
        }
    }
    const double common = r / (2.0 * gamma);
    const double* l2[2] = {lp, lm};
    double* out2[2] = {fpos, fneg};
    for (int s = 0; s < 2; ++s) {
        const double* l = l2[s];
        double* f = out2[s];
        const double W1 = 2.0 * (gamma - 1.0) * l[0] + l[3] + l[4];
        const double W2 = l[3] - l[4];
        const double W3 = l[3] + l[4];
        f[0] = common * W1;
        f[1] = common * (u * W1 + a * n[0] * W2);
        f[2] = common * (v * W1 + a * n[1] * W2);
        f[3] = common * (w * W1 + a * n[2] * W2);
        f[4] = common * (0.5 * q2 * W1 + a * un * W2 + (a * a / (gamma - 1.0)) * W3);
    }
    return SFO_OK;
}

/* StegerWarmingFlux::flux, SF_sw.cpp:22-28: F+(qL) + F-(qR). */
int sfo_steger_flux(const double* qL, const double* qR, const double* n, double gamma, double* out) {
    double fp[5], fm[5], unused[5];
    int err = steger_split(qL, n, gamma, fp, unused);
    if (!err) err = steger_split(qR, n, gamma, unused, fm);
    if (err) return err;
    for (int v = 0; v < 5; ++v) out[v] = fp[v] + fm[v];
    return SFO_OK;
}

/* Riemann::splitLaxFriedrichs, SF_riemann.cpp:125-152: (F +- lam_max Q) / 2
 * with the state's own lam_max = |u.n| + a. */
static int lf_split(const double* Q, const double* n, double gamma, double* fpos, double* fneg) {
    const double r = Q[0];
    double p;
    int err = physical_pressure(Q, gamma, &p);
    if (err) return err;
    const double invR = 1.0 / r;
    const double u = Q[1] * invR, v = Q[2] * invR, w = Q[3] * invR;
    const double a = sqrt(gamma * p * invR);
    const double un = u * n[0] + v * n[1] + w * n[2];
    const double lam_max = fabs(un) + a;
    double F[5];
    F[0] = r * un;
    F[1] = Q[1] * un + p * n[0];
    F[2] = Q[2] * un + p * n[1];
    F[3] = Q[3] * un + p * n[2];
    F[4] = (Q[4] + p) * un;
    for (int i = 0; i < 5; ++i) {
        fpos[i] = 0.5 * (F[i] + lam_max * Q[i]);
        fneg[i] = 0.5 * (F[i] - lam_max * Q[i]);
    }
    return SFO_OK;
}

/* LaxFriedrichsFlux::flux, SF_lxF.cpp: F+(qL) + F-(qR). */
int sfo_lf_flux(const double* qL, const double* qR, const double* n, double gamma, double* out) {
    double fp[5], fm[5], unused[5];
    int err = lf_split(qL, n, gamma, fp, unused);
    if (!err) err = lf_split(qR, n, gamma, unused, fm);
    if (err) return err;
    for (int v = 0; v < 5; ++v) out[v] = fp[v] + fm[v];
    return SFO_OK;
}

/* LaxWendroffFlux::flux, SF_lw.cpp:17-40: the physical flux of the
 * Richtmyer half-step state (qL + qR)/2 - dt/(2 s) (F(qR) - F(qL)), s the
 * face spacing.  dt and s must be > 0 (the reference exits otherwise). */
int sfo_lw_flux(const double* qL, const double* qR, const double* n, double dt, double spacing, double gamma,
                double* out) {
    if (!(dt > 0.0) || !(spacing > 0.0)) return SFO_ERR_ARG;
    double fL[5], fR[5];
    int err = physical_euler_flux(qL, n, gamma, fL);
    if (!err) err = physical_euler_flux(qR, n, gamma, fR);
    if (err) return err;
    const double lambda = dt / spacing;
    double qHalf[5];
    for (int v = 0; v < 5; ++v) qHalf[v] = 0.5 * (qL[v] + qR[v]) - 0.5 * lambda * (fR[v] - fL[v]);
    return physical_euler_flux(qHalf, n, gamma, out);
}

/* ------------------------------------------------------------------ */

static __thread sfo_counters* g_counters = NULL;
/* Step size seen by the Lax-Wendroff flux inside sfo_rhs: set by the stage
 * driver from its dt (divDispatch receives the step's dt the same way). */
static __thread double g_lw_dt = 0.0;

void sfo_set_step_dt(double dt) { g_lw_dt = dt; }
double sfo_step_dt(void) { return g_lw_dt; }

/* characteristicWENOFaceFlux<NStencil>, SF_WENO.h:184-245, with the scalar
 * stencil gather of fillScalarWENOStencils (SF_WENO.h:79-98): the left state
 * reads points 0..w-1 and the right state the mirrored points N-1..N-w. */
int sfo_char_face_flux(int nstencil, const double* stencil, const double* metrics, int scheme,
                       int flux, double gamma, double* out) {
    return sfo_char_face_flux_ex(nstencil, stencil, metrics, scheme, flux, gamma, g_lw_dt, 0.0, out);
}

/* The same with the step size and face spacing the Lax-Wendroff flux needs
 * (Flux::faceSpacing, SF_face.h:92-106). */
int sfo_char_face_flux_ex(int nstencil, const double* stencil, const double* metrics, int scheme,
                          int flux, double gamma, double dt, double spacing, double* out) {
    const int width = nstencil == 4 ? 4 : (nstencil == 6 ? 5 : 7);
    if (!(nstencil == 4 || nstencil == 6 || nstencil == 8)) return SFO_ERR_ARG;
    const double sx = metrics[0], sy = metrics[1], sz = metrics[2];
    const double smag = sqrt(sx * sx + sy * sy + sz * sz);
    if (!isfinite(smag) || smag <= 1.0e-300) return SFO_ERR_ARG;
    const double normal[3] = {sx / smag, sy / smag, sz / smag};
    const double area = smag;
    const int cl = nstencil / 2 - 1;
    double qAvg[5];
    for (int v = 0; v < 5; ++v) qAvg[v] = 0.5 * (stencil[cl * 5 + v] + stencil[(cl + 1) * 5 + v]);
    double L[25], R[25];
    int err = sfo_char_matrix(qAvg, normal, gamma, L, R);
    if (err) return err;
    double ch[8][5];
    for (int s = 0; s < nstencil; ++s) gemv5(L, stencil + s * 5, ch[s]);
    double wL[5], wR[5];
    for (int v = 0; v < 5; ++v) {
        double sl[8] = {0}, sr[8] = {0};
        for (int s = 0; s < width; ++s) {
            sl[s] = ch[s][v];
            sr[s] = ch[nstencil - 1 - s][v];
            if (!isfinite(sl[s]) || !isfinite(sr[s])) return SFO_ERR_NONFINITE;
        }
        switch (scheme) {
        case SFO_WENO3: wL[v] = sfo_weno3_core(sl); wR[v] = sfo_weno3_core(sr); break;
        case SFO_WENO5: wL[v] = sfo_weno5_core(sl); wR[v] = sfo_weno5_core(sr); break;
        case SFO_WENO7: wL[v] = sfo_weno7_core(sl); wR[v] = sfo_weno7_core(sr); break;
        case SFO_TENO5: {
            int ml = 0, mr = 0;
            wL[v] = sfo_teno5_core(sl, &ml);
            wR[v] = sfo_teno5_core(sr, &mr);
            if (g_counters) {
                g_counters->teno_cores += 2;
                g_counters->teno_cut += (unsigned)__builtin_popcount(ml) + (unsigned)__builtin_popcount(mr);
            }
            if (isnan(wL[v]) && ml == 7) return SFO_ERR_TENO_CUTOFF;
            if (isnan(wR[v]) && mr == 7) return SFO_ERR_TENO_CUTOFF;
            break;
        }
        default: return SFO_ERR_ARG;
        }
        if (!isfinite(wL[v]) || !isfinite(wR[v])) return SFO_ERR_NONFINITE;
    }
    double qL[5], qR[5], f[5];
    gemv5(R, wL, qL);
    gemv5(R, wR, qR);
    switch (flux) {
    case SFO_STEGER: err = sfo_steger_flux(qL, qR, normal, gamma, f); break;
    case SFO_RUSANOV: err = sfo_rusanov_flux(qL, qR, normal, gamma, f); break;
    case SFO_LAXFRIEDRICHS: err = sfo_lf_flux(qL, qR, normal, gamma, f); break;
    case SFO_ROE: err = sfo_roe_flux(qL, qR, normal, gamma, f); break;
    case SFO_LAXWENDROFF: err = sfo_lw_flux(qL, qR, normal, dt, spacing, gamma, f); break;
    default: return SFO_ERR_ARG;
    }
    if (err) return err;
    for (int v = 0; v < 5; ++v) out[v] = f[v] * area;
    if (g_counters) g_counters->faces += 1;
    return SFO_OK;
}

/* ------------------------------------------------------------------ */
/* Grid helpers                                                        */
/* ------------------------------------------------------------------ */

typedef struct {
    int m[3];          /* storage extents */
    int lo[3];         /* first interior index per axis */
    long long stride[3];
    double jac;        /* 1/J */
    double metric[3];  /* xi_x, eta_y, zeta_z */
    double area[3];    /* face cofactor magnitude per axis */
} layout;

static void make_layout(const sfo_grid* g, layout* L) {
    for (int d = 0; d < 3; ++d) {
        int active = d < g->dim;
        L->m[d] = g->n[d] + (active ? 2 * g->ng : 0);
        L->lo[d] = active ? g->ng : 0;
    }
    L->stride[0] = NV;
    L->stride[1] = (long long)NV * L->m[0];
    L->stride[2] = (long long)NV * L->m[0] * L->m[1];
    /* Uniform Cartesian metrics as the mesh builds them (SF_mesh.cpp:283-339):
     * J = dx dy dz, Jac = 1/J, xi_x = (dy dz) Jac, ...; face cofactor is the
     * average of metric/Jac on both sides (SF_canonicalFace.h:94-103). */
    const double hx = g->h[0], hy = g->h[1], hz = g->h[2];
    const double J = hx * hy * hz;
    L->jac = 1.0 / J;
    L->metric[0] = (hy * hz) * L->jac;
    L->metric[1] = (hx * hz) * L->jac;
    L->metric[2] = (hx * hy) * L->jac;
    for (int d = 0; d < 3; ++d)
        L->area[d] = 0.5 * (L->metric[d] / L->jac + L->metric[d] / L->jac);
}

long long sfo_storage_size(const sfo_grid* g) {
    layout L;
    make_layout(g, &L);
    return (long long)NV * L.m[0] * L.m[1] * L.m[2];
}

static int grid_ok(const sfo_grid* g) {
    if (g->dim < 1 || g->dim > 3 || g->ng < 2 || g->ng > 4) return 0;
    for (int d = 0; d < 3; ++d) {
        if (g->n[d] < 1) return 0;
        if (d >= g->dim && g->n[d] != 1) return 0;
        if (!(g->h[d] > 0.0)) return 0;
        if (d < g->dim && (g->bc_lo[d] == SFO_BC_LAW || g->bc_hi[d] == SFO_BC_LAW) && (!g->law || g->n[d] < 3))
            return 0;
    }
    return g->gamma > 1.0;
}

static int node_solved(const sfo_grid* g, const layout* L, const int* idx) {
    for (int d = 0; d < g->dim; ++d) {
        int node = idx[d] - L->lo[d];
        if (node == 0 && (g->bc_lo[d] == SFO_BC_TRANSMISSIVE || g->bc_lo[d] == SFO_BC_LAW)) return 0;
        if (node == g->n[d] - 1 && (g->bc_hi[d] == SFO_BC_TRANSMISSIVE || g->bc_hi[d] == SFO_BC_LAW)) return 0;
    }
    return 1;
}

static int fill_laws(const sfo_grid* g, const layout* L, double* Q);

/* Boundary laws (SF_applicator.h:51-83 -> SF_zeroGradient.cpp:88-105 for
 * transmissive; wrap for periodic; nothing for frozen; fill_laws for the
 * per-field laws of LAW ends). */
int sfo_fill_ghosts(const sfo_grid* g, double* Q) {
    if (!grid_ok(g)) return SFO_ERR_ARG;
    layout L;
    make_layout(g, &L);
    const int ng = g->ng;
    for (int d = 0; d < g->dim; ++d) {
        const int n = g->n[d];
        /* iterate over all storage positions of the two other axes */
        int a1 = (d + 1) % 3, a2 = (d + 2) % 3;
        for (int p2 = 0; p2 < L.m[a2]; ++p2)
            for (int p1 = 0; p1 < L.m[a1]; ++p1) {
                long long base = (long long)p1 * L.stride[a1] + (long long)p2 * L.stride[a2];
                const long long sd = L.stride[d];
                double* line = Q + base;
#define AT(ii) (line + (long long)(ii) * sd)
                /* low end */
                if (g->bc_lo[d] == SFO_BC_TRANSMISSIVE) {
                    if (n > 1) memcpy(AT(ng), AT(ng + 1), sizeof(double) * NV);
                    for (int b = 0; b < ng; ++b) memcpy(AT(b), AT(ng), sizeof(double) * NV);
                } else if (g->bc_lo[d] == SFO_BC_PERIODIC) {
                    for (int b = 0; b < ng; ++b) memcpy(AT(b), AT(b + n), sizeof(double) * NV);
                }
                /* high end */
                if (g->bc_hi[d] == SFO_BC_TRANSMISSIVE) {
                    if (n > 1) memcpy(AT(n + ng - 1), AT(n + ng - 2), sizeof(double) * NV);
                    for (int b = 1; b <= ng; ++b)
                        memcpy(AT(n + ng - 1 + b), AT(n + ng - 1), sizeof(double) * NV);
                } else if (g->bc_hi[d] == SFO_BC_PERIODIC) {
                    for (int b = 0; b < ng; ++b) memcpy(AT(n + ng + b), AT(ng + b), sizeof(double) * NV);
                }
#undef AT
            }
    }
    return fill_laws(g, &L, Q);
}

/* ---- Per-field boundary laws of LAW ends -----------------------------------
 * Boundary::Applicator::apply (SF_applicator.h:51-83) runs the density laws of
 * every patch, then the velocity laws, then the pressure laws, each over the
 * points of the patch's set.  Every ghost layer of a point is derived from the
 * boundary node itself (forBoundaryGhostsAlongAxis, SF_boundary.h:95-121).
 *
 * Densities and pressures of some points are read through the Field's
 * thermodynamic state cache (Field::thermodynamicState, SF_field.cpp:133-151;
 * ThermodynamicStateCache, SF_thermodynamicStateCache.h): a direct-mapped
 * table of min(storage points, 4096) entries indexed by the Field cell
 * index.  It is emptied right before the laws run (SF_conservativeRHS.cpp:93)
 * and the laws' own writes do not refresh it, so a state that the velocity
 * fixedValue law caches before it writes the momentum is the state the
 * pressure law later reads for the ghosts.  tcache reproduces that table.
 * The Field of the reference carries ghosts on every axis; ref_cell maps a
 * compact storage position to its cell index there. */

#define SFO_GAS_CONSTANT 287.05  /* makeSingleFluidPerfectGas, fluidStateModel/SF_factory.h:21-33 */
#define SFO_CACHE_MAX 4096       /* Field::setStateModel, SF_field.cpp:117-118 */

typedef struct { long long cell; double rho, p; } tcache_entry;
typedef struct {
    tcache_entry e[SFO_CACHE_MAX];
    long long cap, mx, my;
    int off[3];
    double gamma;
} tcache;

static long long ref_cell(const tcache* c, const int* at) {
    return ((long long)(at[2] + c->off[2]) * c->my + (at[1] + c->off[1])) * c->mx + (at[0] + c->off[0]);
}

/* Field::thermodynamicState: SingleFluidStateModel::close
 * (SF_singleFluidStateModel.cpp:49-73) with PerfectGasEOS::fromDensityEnergy
 * and its checks (SF_perfectGasEOS.h:26-33,80-86), through the cache. */
static int cached_state(tcache* c, const int* at, const double* q, double* rho, double* p) {
    const long long cell = ref_cell(c, at);
    tcache_entry* e = &c->e[cell % c->cap];
    if (e->cell == cell) {
        *rho = e->rho;
        *p = e->p;
        return SFO_OK;
    }
    if (!isfinite(q[0]) || q[0] <= 0.0) return SFO_ERR_STATE;       /* requireEnergyInput */
    for (int d = 1; d < 4; ++d)
        if (!isfinite(q[d])) return SFO_ERR_NONFINITE;
    const double r = q[0];
    double u[3];
    for (int d = 0; d < 3; ++d) u[d] = q[1 + d] / r;
    const double kinetic = 0.5 * r * (u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    const double eint = q[4] - kinetic;
    const double em = eint / r;
    const double thermal = em - 0.0;
    const double pp = (c->gamma - 1.0) * r * thermal;
    const double T = thermal * (c->gamma - 1.0) / SFO_GAS_CONSTANT;
    const double cs = sqrt(c->gamma * pp / r);
    if (!isfinite(em) || !isfinite(pp) || pp <= 0.0 || !isfinite(T) || T <= 0.0 || !isfinite(cs) || cs <= 0.0)
        return SFO_ERR_STATE;
    e->cell = cell;
    e->rho = r;
    e->p = pp;
    *rho = r;
    *p = pp;
    return SFO_OK;
}

/* setEnergyFromPressure (SF_thermodynamicClosure.cpp:166-184) through
 * SingleFluidStateModel::totalEnergyFromPressure / totalEnergyFromThermo
 * (SF_singleFluidStateModel.cpp:75-102) and PerfectGasEOS::fromDensityPressure
 * (SF_perfectGasEOS.h:43-53). */
static int energy_from_pressure(double* q, double gamma, double p) {
    if (!isfinite(p) || p <= 0.0) return SFO_ERR_STATE;
    if (!isfinite(q[0]) || q[0] <= 0.0) return SFO_ERR_STATE;
    for (int d = 1; d < 4; ++d)
        if (!isfinite(q[d])) return SFO_ERR_NONFINITE;
    const double thermal = p / ((gamma - 1.0) * q[0]);
    const double e = 0.0 + thermal;
    const double T = p / (q[0] * SFO_GAS_CONSTANT);
    const double cs = sqrt(gamma * p / q[0]);
    if (!isfinite(e) || !isfinite(T) || T <= 0.0 || !isfinite(cs) || cs <= 0.0) return SFO_ERR_STATE;
    const double inv = 1.0 / q[0];
    const double kinetic = 0.5 * inv * (q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    q[4] = q[0] * e + kinetic;
    return SFO_OK;
}

static int positive_density(const double* q) { return isfinite(q[0]) && q[0] > 0.0; }

/* One family of laws (0 density, 1 velocity, 2 pressure) at one boundary
 * point.  b, s: storage positions of the boundary node and of its inner
 * sample (nearestInsideSample, SF_zeroGradient.cpp:35-52); gp: the ng ghost
 * positions in the reference's visiting order. */
static int law_point(tcache* c, const sfo_law* law, int family, int axis, double gamma, double* Q,
                     const layout* L, const int* b, const int* s, int (*gp)[3], int ng) {
#define PTR(at) (Q + (at)[0] * L->stride[0] + (at)[1] * L->stride[1] + (at)[2] * L->stride[2])
    double* qb = PTR(b);
    const double* qs = PTR(s);
    double rr, pr;
    int err;
    if (family == 0) {
        /* FixedValue::applyScalar (SF_fixedValue.cpp:110-127): ghost = 2 v - q_b;
         * ZeroGradient / Symmetry::applyScalar (SF_zeroGradient.cpp:88-105) */
        if (law->rho == SFO_LAW_FIXED_VALUE) {
            qb[0] = law->rho_value;
            for (int k = 0; k < ng; ++k) PTR(gp[k])[0] = 2.0 * law->rho_value - qb[0];
        } else {
            qb[0] = qs[0];
            for (int k = 0; k < ng; ++k) PTR(gp[k])[0] = qb[0];
        }
        return SFO_OK;
    }
    if (family == 1) {
        if (law->U == SFO_LAW_FIXED_VALUE) {
            /* FixedValue::applyVector3 (SF_fixedValue.cpp:129-160) */
            err = cached_state(c, b, qb, &rr, &pr);
            if (err) return err;
            for (int d = 0; d < 3; ++d) qb[1 + d] = rr * law->U_value[d];
            for (int k = 0; k < ng; ++k) {
                double* qg = PTR(gp[k]);
                double rg, u[3];
                err = cached_state(c, b, qb, &rr, &pr);
                if (err) return err;
                for (int d = 0; d < 3; ++d) u[d] = qb[1 + d] / rr;
                err = cached_state(c, gp[k], qg, &rg, &pr);
                if (err) return err;
                for (int d = 0; d < 3; ++d) qg[1 + d] = rg * (2.0 * law->U_value[d] - u[d]);
            }
        } else if (law->U == SFO_LAW_SYMMETRY) {
            /* Symmetry::applyVector3 (SF_symmetry.cpp:82-136): tangential
             * velocity copied from the inner sample, normal component 0;
             * ghosts mirror the normal component */
            if (!positive_density(qb) || !positive_density(qs)) return SFO_ERR_STATE;
            const double scale = qb[0] / qs[0];
            double v[3];
            for (int d = 0; d < 3; ++d) v[d] = qs[1 + d] * scale;
            v[axis] = 0.0;
            for (int d = 0; d < 3; ++d) qb[1 + d] = v[d];
            for (int k = 0; k < ng; ++k) {
                double* qg = PTR(gp[k]);
                double m[3];
                for (int d = 0; d < 3; ++d) m[d] = qb[1 + d];
                m[axis] = -m[axis];
                if (!positive_density(qg) || !positive_density(qb)) return SFO_ERR_STATE;
                const double sg = qg[0] / qb[0];
                for (int d = 0; d < 3; ++d) qg[1 + d] = m[d] * sg;
            }
        } else {
            /* ZeroGradient::applyVector3 (SF_zeroGradient.cpp:107-131) */
            for (int d = 1; d < 4; ++d) qb[d] = qs[d];
            for (int k = 0; k < ng; ++k)
                for (int d = 1; d < 4; ++d) PTR(gp[k])[d] = qb[d];
        }
        return SFO_OK;
    }
    /* updateEnergyFromPressure (SF_thermodynamicClosure.cpp:219-285) */
    if (law->p == SFO_LAW_FIXED_VALUE) {
        err = energy_from_pressure(qb, gamma, law->p_value);
        if (err) return err;
        for (int k = 0; k < ng; ++k) {
            err = cached_state(c, b, qb, &rr, &pr);
            if (err) return err;
            err = energy_from_pressure(PTR(gp[k]), gamma, 2.0 * law->p_value - pr);
            if (err) return err;
        }
    } else {
        double rs, ps;
        err = cached_state(c, s, qs, &rs, &ps);
        if (err) return err;
        err = energy_from_pressure(qb, gamma, ps);
        if (err) return err;
        for (int k = 0; k < ng; ++k) {
            err = cached_state(c, b, qb, &rr, &pr);
            if (err) return err;
            err = energy_from_pressure(PTR(gp[k]), gamma, pr);
            if (err) return err;
        }
    }
    return SFO_OK;
#undef PTR
}

/* The laws of every LAW end: density for all ends, then velocity, then
 * pressure; ends in the order x low, x high, y low, ...; the points of an
 * end's face with the last axis outermost. */
static int fill_laws(const sfo_grid* g, const layout* L, double* Q) {
    int any = 0;
    for (int d = 0; d < g->dim; ++d) any |= g->bc_lo[d] == SFO_BC_LAW || g->bc_hi[d] == SFO_BC_LAW;
    if (!any) return SFO_OK;
    tcache* c = (tcache*)malloc(sizeof(tcache));
    if (!c) return SFO_ERR_ARG;
    const int ng = g->ng;
    c->mx = g->n[0] + 2 * ng;
    c->my = g->n[1] + 2 * ng;
    const long long total = c->mx * c->my * (long long)(g->n[2] + 2 * ng);
    c->cap = total < SFO_CACHE_MAX ? total : SFO_CACHE_MAX;
    for (int d = 0; d < 3; ++d) c->off[d] = d < g->dim ? 0 : ng;
    c->gamma = g->gamma;
    for (long long i = 0; i < c->cap; ++i) c->e[i].cell = -1;
    int err = SFO_OK;
    for (int family = 0; family < 3 && !err; ++family)
        for (int axis = 0; axis < g->dim && !err; ++axis)
            for (int end = 0; end < 2 && !err; ++end) {
                if ((end ? g->bc_hi[axis] : g->bc_lo[axis]) != SFO_BC_LAW) continue;
                const sfo_law* law = &g->law[2 * axis + end];
                const int n = g->n[axis];
                const int bnode = end ? n - 1 : 0, snode = end ? n - 2 : 1;
                int node[3];
                for (node[2] = 0; node[2] < g->n[2] && !err; ++node[2])
                    for (node[1] = 0; node[1] < g->n[1] && !err; ++node[1])
                        for (node[0] = 0; node[0] < g->n[0] && !err; ++node[0]) {
                            if (node[axis] != bnode) continue;
                            int b[3], s[3], gp[4][3];
                            for (int d = 0; d < 3; ++d) b[d] = s[d] = L->lo[d] + node[d];
                            s[axis] = L->lo[axis] + snode;
                            for (int k = 0; k < ng; ++k) {
                                for (int d = 0; d < 3; ++d) gp[k][d] = b[d];
                                gp[k][axis] = end ? b[axis] + 1 + k : k;
                            }
                            err = law_point(c, law, family, axis, g->gamma, Q, L, b, s, gp, ng);
                        }
            }
    free(c);
    return err;
}

static int stencil_points(int scheme) {
    return scheme == SFO_WENO3 ? 4 : (scheme == SFO_WENO7 ? 8 : 6);
}

/* Face loops of forFaces (SF_iteration.h:60-82) + storeFlux and residual
 * assembly (SF_faceAssembly.h:26-88, SF_residualAssembly.h:12-32). */
int sfo_rhs(const sfo_grid* g, int scheme, int flux, const double* Q, double* R, sfo_counters* counters) {
    if (!grid_ok(g)) return SFO_ERR_ARG;
    const int nst = stencil_points(scheme);
    if (g->ng < nst / 2) return SFO_ERR_ARG;    /* checkGhostDepth, SF_stencil.h:23-34 */
    layout L;
    make_layout(g, &L);
    const long long total = (long long)L.m[0] * L.m[1] * L.m[2];
    double* F[3] = {NULL, NULL, NULL};
    int err = SFO_OK;
    g_counters = counters;
    for (int d = 0; d < g->dim; ++d) {
        F[d] = (double*)calloc((size_t)total * NV, sizeof(double));
        if (!F[d]) { err = SFO_ERR_ARG; goto done; }
    }
    if (g->metrics && flux == SFO_LAXWENDROFF) { err = SFO_ERR_ARG; goto done; }  /* needs coordinates */
    for (int d = 0; d < g->dim && !err; ++d) {
        double metrics[4] = {d == 0 ? L.area[0] : 0.0, d == 1 ? L.area[1] : 0.0,
                             d == 2 ? L.area[2] : 0.0, L.jac};
        int lo[3], hi[3];
        for (int a = 0; a < 3; ++a) {
            lo[a] = L.lo[a];
            hi[a] = L.lo[a] + g->n[a];
        }
        lo[d] -= 1;  /* faces i+1/2 for i in [ng-1, n+ng-1] */
        const long long sd = L.stride[d];
        for (int k = lo[2]; k < hi[2] && !err; ++k)
            for (int j = lo[1]; j < hi[1] && !err; ++j)
                for (int i = lo[0]; i < hi[0]; ++i) {
                    const long long at = i * L.stride[0] + j * L.stride[1] + k * L.stride[2];
                    double st[8 * 5];
                    for (int s = 0; s < nst; ++s) {
                        const long long off = at + (long long)(s - (nst / 2 - 1)) * sd;
                        for (int v = 0; v < 5; ++v) st[s * 5 + v] = Q[off + v];
                    }
                    /* faceSpacing on coordinates X = (index - ng) h, as the
                     * reference Field of the harness holds them */
                    const int li = d == 0 ? i : (d == 1 ? j : k);
                    const double xl = (double)(li - g->ng) * g->h[d], xr = (double)(li + 1 - g->ng) * g->h[d];
                    double spacing = fabs(xr - xl);
                    spacing = spacing > 1e-14 ? spacing : 1e-14;
                    double f[5];
                    if (g->metrics) {
                        /* canonicalFace::geometry without stored face metrics
                         * (SF_canonicalFace.h:56-118): the cofactor averaged
                         * from metricCofactor(m, Jac) = m / Jac of both nodes */
                        const long long pa = at / NV, pb = (at + sd) / NV;
                        const double* ma = g->metrics + pa * 10;
                        const double* mb = g->metrics + pb * 10;
                        if (!isfinite(ma[0]) || !isfinite(mb[0]) || fabs(ma[0]) < 1.0e-30 || fabs(mb[0]) < 1.0e-30) {
                            err = SFO_ERR_ARG;
                            break;
                        }
                        for (int c = 0; c < 3; ++c)
                            metrics[c] = 0.5 * (ma[1 + 3 * d + c] / ma[0] + mb[1 + 3 * d + c] / mb[0]);
                        metrics[3] = 0.5 * (ma[0] + mb[0]);
                    }
                    err = sfo_char_face_flux_ex(nst, st, metrics, scheme, flux, g->gamma, g_lw_dt, spacing, f);
                    if (err) break;
                    for (int v = 0; v < 5; ++v) {
                        if (!isfinite(f[v])) { err = SFO_ERR_NONFINITE; break; }
                        F[d][at + v] = f[v];
                    }
                    if (err) break;
                }
    }
    if (err) goto done;
    memset(R, 0, sizeof(double) * (size_t)total * NV);
    for (int k = L.lo[2]; k < L.lo[2] + g->n[2]; ++k)
        for (int j = L.lo[1]; j < L.lo[1] + g->n[1]; ++j)
            for (int i = L.lo[0]; i < L.lo[0] + g->n[0]; ++i) {
                const long long at = i * L.stride[0] + j * L.stride[1] + k * L.stride[2];
                const double jac = g->metrics ? g->metrics[(at / NV) * 10] : L.jac;
                for (int v = 0; v < 5; ++v) {
                    double div = 0.0;
                    for (int d = 0; d < g->dim; ++d)
                        div += F[d][at + v] - F[d][at - L.stride[d] + v];
                    R[at + v] = jac * div - 0.0;
                }
            }
done:
    g_counters = NULL;
    for (int d = 0; d < 3; ++d) free(F[d]);
    return err;
}

/* RusanovEOS::deltaT, SF_rusanovEOS.cpp:110-147 over forFluidInterior. */
int sfo_dt(const sfo_grid* g, const double* Q, double cfl, double* dt) {
    if (!grid_ok(g) || !isfinite(cfl) || cfl <= 0.0) return SFO_ERR_ARG;
    layout L;
    make_layout(g, &L);
    double result = 1.7976931348623157e308;
    int idx[3];
    for (idx[2] = L.lo[2]; idx[2] < L.lo[2] + g->n[2]; ++idx[2])
        for (idx[1] = L.lo[1]; idx[1] < L.lo[1] + g->n[1]; ++idx[1])
            for (idx[0] = L.lo[0]; idx[0] < L.lo[0] + g->n[0]; ++idx[0]) {
                if (!node_solved(g, &L, idx)) continue;
                const double* q = Q + idx[0] * L.stride[0] + idx[1] * L.stride[1] + idx[2] * L.stride[2];
                closed_state s;
                int err = close_state(q, g->gamma, &s);
                if (err) return err;
                /* metric vectors: per node on curvilinear grids, else
                 * (xi_x,0,0), (0,eta_y,0), (0,0,zeta_z) */
                double mv[9] = {L.metric[0], 0.0, 0.0, 0.0, L.metric[1], 0.0, 0.0, 0.0, L.metric[2]};
                if (g->metrics) {
                    const double* m = g->metrics + ((idx[0] * L.stride[0] + idx[1] * L.stride[1] + idx[2] * L.stride[2]) / NV) * 10;
                    for (int c = 0; c < 9; ++c) mv[c] = m[1 + c];
                }
                const double ux = fabs(s.vel[0] * mv[0] + s.vel[1] * mv[1] + s.vel[2] * mv[2]);
                const double ue = fabs(s.vel[0] * mv[3] + s.vel[1] * mv[4] + s.vel[2] * mv[5]);
                const double uz = fabs(s.vel[0] * mv[6] + s.vel[1] * mv[7] + s.vel[2] * mv[8]);
                double sr = 0.0;
                if (g->dim > 0) sr += ux + s.c * sqrt(mv[0] * mv[0] + mv[1] * mv[1] + mv[2] * mv[2]);
                if (g->dim > 1) sr += ue + s.c * sqrt(mv[3] * mv[3] + mv[4] * mv[4] + mv[5] * mv[5]);
                if (g->dim > 2) sr += uz + s.c * sqrt(mv[6] * mv[6] + mv[7] * mv[7] + mv[8] * mv[8]);
                if (!isfinite(sr) || sr <= 0.0) return SFO_ERR_STATE;
                const double cand = cfl / sr;
                if (cand < result) result = cand;
            }
    *dt = result;
    return SFO_OK;
}

/* Post-update state validation (validateEquationState / applyDivergence's
 * requirePhysicalState): rho > 0, p > 0, finite. */
static int validate_solved(const sfo_grid* g, const layout* L, const double* Q) {
    int idx[3];
    for (idx[2] = L->lo[2]; idx[2] < L->lo[2] + g->n[2]; ++idx[2])
        for (idx[1] = L->lo[1]; idx[1] < L->lo[1] + g->n[1]; ++idx[1])
            for (idx[0] = L->lo[0]; idx[0] < L->lo[0] + g->n[0]; ++idx[0]) {
                if (!node_solved(g, L, idx)) continue;
                const double* q = Q + idx[0] * L->stride[0] + idx[1] * L->stride[1] + idx[2] * L->stride[2];
                double p;
                int err = physical_pressure(q, g->gamma, &p);
                if (err) return err;
            }
    return SFO_OK;
}

static int stage_count(int time_id) {
    return time_id == SFO_EULER ? 1 : (time_id == SFO_SSPRK3 ? 3 : (time_id == SFO_RK4 ? 4 : 0));
}

/* One stage of Time::Explicit::executeStage (SF_explicit.cpp:331-530) with
 * the Shu-Osher / RK4 tableaux of SF_builtinProviders.cpp:84-126.
 * work layout: [q0 | R | k1 | k2 | k3] each storage-size doubles (k4 = R). */
int sfo_stage_fn(const sfo_grid* g, sfo_rhs_fn rhs, void* ctx, int time_id, double* Q, double dt,
                 int stage, double* work) {
    const int ns = stage_count(time_id);
    if (!ns || stage < 0 || stage >= ns) return SFO_ERR_ARG;
    g_lw_dt = dt;  /* the spatial operator of this stage sees the step's dt */
    layout L;
    make_layout(g, &L);
    const long long S = sfo_storage_size(g);
    double* q0 = work;
    double* Rr = work + S;
    double* k1 = work + 2 * S;
    double* k2 = work + 3 * S;
    double* k3 = work + 4 * S;
    int err;
    if (stage == 0 && time_id != SFO_EULER) {
        /* Explicit::begin snapshots q0 on solved nodes (SF_explicit.cpp:171-179) */
        memset(q0, 0, sizeof(double) * (size_t)S);
        int idx[3];
        for (idx[2] = L.lo[2]; idx[2] < L.lo[2] + g->n[2]; ++idx[2])
            for (idx[1] = L.lo[1]; idx[1] < L.lo[1] + g->n[1]; ++idx[1])
                for (idx[0] = L.lo[0]; idx[0] < L.lo[0] + g->n[0]; ++idx[0]) {
                    if (!node_solved(g, &L, idx)) continue;
                    long long at = idx[0] * L.stride[0] + idx[1] * L.stride[1] + idx[2] * L.stride[2];
                    memcpy(q0 + at, Q + at, sizeof(double) * NV);
                }
    }
    err = sfo_fill_ghosts(g, Q);   /* prepareBoundaryState before the RHS */
    if (err) return err;
    err = rhs(ctx, Q, Rr);
    if (err) return err;
    static const double ssp_base[3] = {0.0, 0.75, 1.0 / 3.0};
    static const double ssp_inc[3] = {1.0, 0.25, 2.0 / 3.0};
    static const double rk4_inc[4] = {0.5, 0.5, 1.0, 0.0};
    int idx[3];
    for (idx[2] = L.lo[2]; idx[2] < L.lo[2] + g->n[2]; ++idx[2])
        for (idx[1] = L.lo[1]; idx[1] < L.lo[1] + g->n[1]; ++idx[1])
            for (idx[0] = L.lo[0]; idx[0] < L.lo[0] + g->n[0]; ++idx[0]) {
                if (!node_solved(g, &L, idx)) continue;
                long long at = idx[0] * L.stride[0] + idx[1] * L.stride[1] + idx[2] * L.stride[2];
                for (int v = 0; v < NV; ++v) {
                    const long long x = at + v;
                    if (time_id == SFO_EULER) {
                        Q[x] -= dt * Rr[x];                                /* applyDivergence */
                    } else if (time_id == SFO_SSPRK3) {
                        const double euler = Q[x] - dt * Rr[x];            /* applySSPStage */
                        Q[x] = ssp_base[stage] * q0[x] + ssp_inc[stage] * euler;
                    } else {
                        if (stage == 0) k1[x] = Rr[x];
                        else if (stage == 1) k2[x] = Rr[x];
                        else if (stage == 2) k3[x] = Rr[x];
                        if (stage < 3) {
                            const double kn = stage == 0 ? k1[x] : (stage == 1 ? k2[x] : k3[x]);
                            Q[x] = q0[x] - rk4_inc[stage] * dt * kn;        /* applyStage */
                        } else {                                           /* applyFinalRK4 */
                            Q[x] = q0[x] - dt / 6.0 * (1.0 * k1[x] + 2.0 * k2[x] + 2.0 * k3[x] + 1.0 * Rr[x]);
                        }
                    }
                }
            }
    err = validate_solved(g, &L, Q);
    if (err) return err;
    if (stage == ns - 1) err = sfo_fill_ghosts(g, Q);  /* FlowStepCommit */
    return err;
}

typedef struct { const sfo_grid* g; int scheme, flux; sfo_counters* counters; } own_ctx;

static int own_rhs(void* c, const double* Q, double* R) {
    own_ctx* o = (own_ctx*)c;
    return sfo_rhs(o->g, o->scheme, o->flux, Q, R, o->counters);
}

static int own_dt(void* c, const double* Q, double cfl, double* dt) {
    own_ctx* o = (own_ctx*)c;
    return sfo_dt(o->g, Q, cfl, dt);
}

int sfo_stage(const sfo_grid* g, int scheme, int flux, int time_id, double* Q, double dt, int stage,
              double* work, sfo_counters* counters) {
    own_ctx o = {g, scheme, flux, counters};
    return sfo_stage_fn(g, own_rhs, &o, time_id, Q, dt, stage, work);
}

int sfo_step(const sfo_grid* g, int scheme, int flux, int time_id, double* Q, double dt, double* work,
             sfo_counters* counters) {
    const int ns = stage_count(time_id);
    if (!ns) return SFO_ERR_ARG;
    int err = sfo_fill_ghosts(g, Q);   /* FlowStepPrepare (SF_flowOperations.cpp:471-485) */
    if (err) return err;
    for (int s = 0; s < ns; ++s) {
        err = sfo_stage(g, scheme, flux, time_id, Q, dt, s, work, counters);
        if (err) return err;
    }
    return SFO_OK;
}

int sfo_advance(const sfo_grid* g, int scheme, int flux, int time_id, double* Q, double t_start,
                double t_end, double cfl, double max_dt, double write_interval, int max_steps,
                double* dt_out, int* steps_done, double* t_final, sfo_counters* counters) {
    own_ctx o = {g, scheme, flux, counters};
    return sfo_advance_fn(g, own_rhs, own_dt, &o, time_id, Q, t_start, t_end, cfl, max_dt,
                          write_interval, max_steps, dt_out, steps_done, t_final);
}

int sfo_advance_fn(const sfo_grid* g, sfo_rhs_fn rhs, sfo_dt_fn dtf, void* ctx, int time_id,
                   double* Q, double t_start, double t_end, double cfl, double max_dt,
                   double write_interval, int max_steps, double* dt_out, int* steps_done,
                   double* t_final) {
    const int ns = stage_count(time_id);
    if (!ns) return SFO_ERR_ARG;
    const long long S = sfo_storage_size(g);
    double* work = (double*)calloc((size_t)S * 5, sizeof(double));
    if (!work) return SFO_ERR_ARG;
    double time = t_start;
    double next_out = write_interval > 0.0 ? t_start + write_interval : INFINITY;
    int step = 0, err = SFO_OK;
    const double eps = 2.220446049250313e-16;
    while (!err) {
        const double remaining = t_end - time;
        double scale = fabs(time) > fabs(t_end) ? fabs(time) : fabs(t_end);
        if (scale < 1.0) scale = 1.0;
        if (remaining <= 64.0 * eps * scale) break;          /* endTimeRoundoffTolerance */
        if (step >= max_steps) break;
        double limit = remaining;
        if (write_interval > 0.0 && next_out - time < limit) limit = next_out - time;
        /* every step opens with FlowStepPrepare (SF_flowOperations.cpp:471-485;
         * the explicit fragment, SF_builtinProviders.cpp:63-81) */
        err = sfo_fill_ghosts(g, Q);
        if (err) break;
        double dt;
        err = dtf(ctx, Q, cfl, &dt);
        if (err) break;
        if (max_dt < dt) dt = max_dt;                         /* std::min({dt, maxDeltaT, limit}) */
        if (limit < dt) dt = limit;
        for (int s = 0; s < ns && !err; ++s) err = sfo_stage_fn(g, rhs, ctx, time_id, Q, dt, s, work);
        if (err) break;
        time += dt;
        if (dt_out) dt_out[step] = dt;
        ++step;
        double sc2 = fabs(time);
        if (sc2 < 1.0) sc2 = 1.0;
        const double tol = 1.0e-11 * sc2;
        if (write_interval > 0.0 && time >= next_out - tol) next_out += write_interval;
    }
    free(work);
    *steps_done = step;
    *t_final = time;
    return err;
}
