// sfg_math.cuh -- device arithmetic of the explicit Euler path.
//
// The reference evaluates every face with dense 5x5 eigenvector matrices built
// for an arbitrary unit normal (src/methods/numerics/convection/SF_riemann.cpp:69-123)
// and 7 divisions per scalar WENO5 core (SF_WENO5.cpp:42-62).  On a Cartesian
// grid the face normal is an axis unit vector, so the tangent basis the
// reference builds is a fixed signed permutation of (x, y, z):
//   normal e_x: l = (-0, 1, 0), m = (0, 0, 1)
//   normal e_y: l = (-1, 0, 0), m = (0, 0, 1)
//   normal e_z: l = (-1, 0, 0), m = (0, -1, 0)
// and L, R collapse to a handful of scalar coefficients.  The functions below
// are the same mathematics with that sparsity folded in; results agree with
// the reference to rounding (the parity tests bound the difference).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "sfg_internal.h"

namespace sfg {

template <int SCHEME> struct SchemeInfo;
template <> struct SchemeInfo<WENO3> { static constexpr int NST = 4, W = 4; };
template <> struct SchemeInfo<WENO5> { static constexpr int NST = 6, W = 5; };
template <> struct SchemeInfo<TENO5> { static constexpr int NST = 6, W = 5; };
template <> struct SchemeInfo<WENO7> { static constexpr int NST = 8, W = 7; };

// Momentum slots (1 + x/y/z) of the normal n and tangents l, m per axis, with
// the sign of the tangent along that slot.
template <int AX> struct AxisBasis;
template <> struct AxisBasis<0> { static constexpr int N = 1, L = 2, M = 3; static constexpr int SL = 1, SM = 1; };
template <> struct AxisBasis<1> { static constexpr int N = 2, L = 1, M = 3; static constexpr int SL = -1, SM = 1; };
template <> struct AxisBasis<2> { static constexpr int N = 3, L = 1, M = 2; static constexpr int SL = -1, SM = -1; };

// FP32 reciprocal as the single SFU instruction (PTX rcp.approx.ftz.f32,
// about 1 ulp).  Every FP32 reciprocal of the path multiplies a deviation or
// feeds a weight ratio, where 1 ulp is below the FP32 rounding already there.
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

template <typename T> __device__ __forceinline__ T rcp(T x);
template <> __device__ __forceinline__ double rcp<double>(double x) { return 1.0 / x; }
template <> __device__ __forceinline__ float rcp<float>(float x) { return rcp_approx(x); }

// ---------------------------------------------------------------------------
// Paired FP32 arithmetic (sm_100 f32x2: one instruction, two lanes of work).
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 swap2(float2 a) { return make_float2(a.y, a.x); }
__device__ __forceinline__ float2 rcp2(float2 a) { return make_float2(rcp_approx(a.x), rcp_approx(a.y)); }

// 1.0f where a >= b, else 0.0f (also for NaN operands): PTX set with a
// floating-point destination, one instruction instead of a compare and a
// select.
__device__ __forceinline__ float ge_one(float a, float b) {
    float r;
    asm("set.ge.f32.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
    return r;
}

// Non-finite watch over a face's paired FP32 work: bad + x * 0 stays exactly
// 0 while every x is finite and turns NaN after an inf or a NaN, one paired
// FMA per watched value and one test per face (flag_bad).
__device__ __forceinline__ float2 watch2(float2 bad, float2 x) { return __ffma2_rn(x, make_float2(0.f, 0.f), bad); }
__device__ __forceinline__ void flag_bad(float2 bad, unsigned& flags) {
    if (!(bad.x == 0.f && bad.y == 0.f)) flags |= FLAG_NONFINITE;
}

template <typename T> __device__ __forceinline__ T div_(T a, T b);
template <> __device__ __forceinline__ double div_<double>(double a, double b) { return a / b; }
template <> __device__ __forceinline__ float div_<float>(float a, float b) { return __fdividef(a, b); }

template <typename T> __device__ __forceinline__ T rsqrt_(T x);
template <> __device__ __forceinline__ double rsqrt_<double>(double x) { return rsqrt(x); }
template <> __device__ __forceinline__ float rsqrt_<float>(float x) { return rsqrtf(x); }

template <typename T> __device__ __forceinline__ T sqrt_(T x);
template <> __device__ __forceinline__ double sqrt_<double>(double x) { return sqrt(x); }
template <> __device__ __forceinline__ float sqrt_<float>(float x) { return sqrtf(x); }

template <typename T> __device__ __forceinline__ bool finite_(T x) { return isfinite(x); }

// ---------------------------------------------------------------------------
// Eigen-structure of the Euler flux Jacobian at the face-average state
// (buildCharacteristicMatrix, SF_riemann.cpp:69-123) in compact form:
//   A = u.m - E - h rho          B = u_n rho - m_n
//   w0 = rho + b1 A   w1 = m_l - u_l rho   w2 = m_m - u_m rho
//   w3 =  x1 B - b2 A              w4 = -x1 B - b2 A
// with h = |u|^2 / 2, b1 = (gamma - 1) / c^2, b2 = b1 / 2, x1 = 1 / (2c), and
// back-projection q = R w:
//   S = w0 + w3 + w4, D = w4 - w3
//   rho = S, m = u S + l w1 + m w2 + c n D, E = h w0 + u_l w1 + u_m w2 + H (w3 + w4) + c u_n D.
// ---------------------------------------------------------------------------
template <typename T> struct Eigen {
    T u, v, w;          // velocity
    T un, ul, um;       // velocity along n, l, m
    T h, H, c, b1, b2, x1;
};

template <int AX, typename T>
__device__ __forceinline__ bool eigen_at(const T q[5], T gamma, Eigen<T>& e) {
    using B = AxisBasis<AX>;
    const T rho = q[0];
    const T inv = rcp<T>(rho);
    e.u = q[1] * inv;
    e.v = q[2] * inv;
    e.w = q[3] * inv;
    const T ke = T(0.5) * (q[1] * q[1] + q[2] * q[2] + q[3] * q[3]) * inv;
    const T p = (gamma - T(1)) * (q[4] - ke);
    const T vel[3] = {e.u, e.v, e.w};
    e.un = vel[B::N - 1];
    e.ul = T(B::SL) * vel[B::L - 1];
    e.um = T(B::SM) * vel[B::M - 1];
    e.h = T(0.5) * (e.u * e.u + e.v * e.v + e.w * e.w);
    e.H = (q[4] + p) * inv;
    const T c2 = gamma * p * inv;
    const T ic = rsqrt_<T>(c2);
    e.c = c2 * ic;
    e.b1 = (gamma - T(1)) * (ic * ic);
    e.b2 = T(0.5) * e.b1;
    e.x1 = T(0.5) * ic;
    return rho > T(0) && p > T(0);
}

template <int AX, typename T>
__device__ __forceinline__ void to_characteristic(const Eigen<T>& e, const T q[5], T w[5]) {
    using B = AxisBasis<AX>;
    const T mn = q[B::N], ml = T(B::SL) * q[B::L], mm = T(B::SM) * q[B::M];
    const T A = e.u * q[1] + e.v * q[2] + e.w * q[3] - q[4] - e.h * q[0];
    const T Bv = e.un * q[0] - mn;
    const T y = e.b2 * A;
    w[0] = q[0] + e.b1 * A;
    w[1] = ml - e.ul * q[0];
    w[2] = mm - e.um * q[0];
    w[3] = e.x1 * Bv - y;
    w[4] = -e.x1 * Bv - y;
}

template <int AX, typename T>
__device__ __forceinline__ void from_characteristic(const Eigen<T>& e, const T w[5], T q[5]) {
    using B = AxisBasis<AX>;
    const T S = w[0] + w[3] + w[4];
    const T D = w[4] - w[3];
    const T cD = e.c * D;
    q[0] = S;
    q[1] = e.u * S;
    q[2] = e.v * S;
    q[3] = e.w * S;
    q[B::N] += cD;
    q[B::L] += T(B::SL) * w[1];
    q[B::M] += T(B::SM) * w[2];
    q[4] = e.h * w[0] + e.ul * w[1] + e.um * w[2] + e.H * (w[3] + w[4]) + e.un * cD;
}

// ---------------------------------------------------------------------------
// Scalar reconstruction cores.  v[0..W-1] is the upwind-ordered stencil.
// ---------------------------------------------------------------------------

// WENO5-JS (SF_WENO5.cpp:42-62): weights d_k/(eps+b_k)^2 normalised.  The
// three alpha divisions and the normalisation are folded into one division:
// with s_k = (eps+b_k)^2, w_k = d_k * prod_{j!=k} s_j, result = sum w_k p_k / sum w_k.
template <typename T>
__device__ __forceinline__ T weno5_core(const T* v, unsigned& flags) {
    const T p0 = T(2) * v[0] - T(7) * v[1] + T(11) * v[2];
    const T p1 = -v[1] + T(5) * v[2] + T(2) * v[3];
    const T p2 = T(2) * v[2] + T(5) * v[3] - v[4];
    const T t0 = v[0] - T(2) * v[1] + v[2], r0 = v[0] - T(4) * v[1] + T(3) * v[2];
    const T t1 = v[1] - T(2) * v[2] + v[3], r1 = v[1] - v[3];
    const T t2 = v[2] - T(2) * v[3] + v[4], r2 = T(3) * v[2] - T(4) * v[3] + v[4];
    const T c13 = T(13.0 / 12.0);
    const T b0 = c13 * (t0 * t0) + T(0.25) * (r0 * r0);
    const T b1 = c13 * (t1 * t1) + T(0.25) * (r1 * r1);
    const T b2 = c13 * (t2 * t2) + T(0.25) * (r2 * r2);
    const T eps = T(1e-6);
    const T s0 = (eps + b0) * (eps + b0);
    const T s1 = (eps + b1) * (eps + b1);
    const T s2 = (eps + b2) * (eps + b2);
    const T w0 = T(0.1) * (s1 * s2);
    const T w1 = T(0.6) * (s0 * s2);
    const T w2 = T(0.3) * (s0 * s1);
    const T den = w0 + w1 + w2;
    if (!(den > T(0)) || !finite_(den)) flags |= FLAG_NONFINITE;
    return div_<T>(w0 * p0 + w1 * p1 + w2 * p2, T(6) * den);
}

// WENO3-JS (SF_WENO3.cpp:42-57), same folding.
template <typename T>
__device__ __forceinline__ T weno3_core(const T* v, unsigned& flags) {
    const T p0 = -v[0] + T(5) * v[1] + T(2) * v[2];
    const T p1 = T(2) * v[1] + T(5) * v[2] - v[3];
    const T b0 = (v[2] - v[0]) * (v[2] - v[0]);
    const T b1 = (v[3] - v[1]) * (v[3] - v[1]);
    const T eps = T(1e-6);
    const T s0 = (eps + b0) * (eps + b0);
    const T s1 = (eps + b1) * (eps + b1);
    const T w0 = T(1.0 / 3.0) * s1;
    const T w1 = T(2.0 / 3.0) * s0;
    const T den = w0 + w1;
    if (!(den > T(0)) || !finite_(den)) flags |= FLAG_NONFINITE;
    return div_<T>(w0 * p0 + w1 * p1, T(6) * den);
}

// Smoothness indicator of a 4-point sub-stencil of WENO7 (SF_WENO7.cpp:41-69):
// the integral over [a, b] of the squared derivatives of the interpolating
// cubic, with the integrals of x^k precomputed per sub-stencil.
template <typename T>
__device__ __forceinline__ T beta4(T v0, T v1, T v2, T v3, T i1, T i2, T i3, T i4, T i5) {
    const T d1 = v1 - v0;
    const T d2 = (v2 - T(2) * v1 + v0) * T(0.5);
    const T d3 = (v3 - T(3) * v2 + T(3) * v1 - v0) * T(1.0 / 6.0);
    const T A = d1 - d2 + T(2) * d3;
    const T Bc = T(2) * d2 - T(6) * d3;
    const T C = T(3) * d3;
    const T beta1 = A * A * i1 + A * Bc * i2 + (Bc * Bc + T(2) * A * C) * i3 + Bc * C * i4 + C * C * i5;
    const T E = T(6) * d3;
    const T beta2 = Bc * Bc * i1 + Bc * E * i2 + E * E * i3;
    const T beta3 = T(36) * d3 * d3 * i1;
    return beta1 + beta2 + beta3;
}

// WENO7-JS (SF_WENO7.cpp:71-98).
template <typename T>
__device__ __forceinline__ T weno7_core(const T* v, unsigned& flags) {
    const T p0 = -T(3) * v[0] + T(13) * v[1] - T(23) * v[2] + T(25) * v[3];
    const T p1 = v[1] - T(5) * v[2] + T(13) * v[3] + T(3) * v[4];
    const T p2 = -v[2] + T(7) * v[3] + T(7) * v[4] - v[5];
    const T p3 = T(3) * v[3] + T(13) * v[4] - T(5) * v[5] + v[6];
    // integrals over [a,b] of 1, x, x^2/3... as used by beta4: b-a, b^2-a^2,
    // (b^3-a^3)/3, (b^4-a^4)/2, (b^5-a^5)/5 for [2.5,3.5], [1.5,2.5], [0.5,1.5], [-0.5,0.5]
    const T b0 = beta4<T>(v[0], v[1], v[2], v[3], T(1), T(6), T(109.0 / 12.0 * 1.0), T(3.5 * 3.5 * 3.5 * 3.5 / 2.0 - 2.5 * 2.5 * 2.5 * 2.5 / 2.0),
                          T((3.5 * 3.5 * 3.5 * 3.5 * 3.5 - 2.5 * 2.5 * 2.5 * 2.5 * 2.5) / 5.0));
    const T b1 = beta4<T>(v[1], v[2], v[3], v[4], T(1), T(4), T(49.0 / 12.0), T(2.5 * 2.5 * 2.5 * 2.5 / 2.0 - 1.5 * 1.5 * 1.5 * 1.5 / 2.0),
                          T((2.5 * 2.5 * 2.5 * 2.5 * 2.5 - 1.5 * 1.5 * 1.5 * 1.5 * 1.5) / 5.0));
    const T b2 = beta4<T>(v[2], v[3], v[4], v[5], T(1), T(2), T(13.0 / 12.0), T(1.5 * 1.5 * 1.5 * 1.5 / 2.0 - 0.5 * 0.5 * 0.5 * 0.5 / 2.0),
                          T((1.5 * 1.5 * 1.5 * 1.5 * 1.5 - 0.5 * 0.5 * 0.5 * 0.5 * 0.5) / 5.0));
    const T b3 = beta4<T>(v[3], v[4], v[5], v[6], T(1), T(0), T(1.0 / 12.0), T(0),
                          T((0.5 * 0.5 * 0.5 * 0.5 * 0.5 + 0.5 * 0.5 * 0.5 * 0.5 * 0.5) / 5.0));
    const T eps = T(1e-6);
    const T a0 = div_<T>(T(1.0 / 35.0), (eps + b0) * (eps + b0));
    const T a1 = div_<T>(T(12.0 / 35.0), (eps + b1) * (eps + b1));
    const T a2 = div_<T>(T(18.0 / 35.0), (eps + b2) * (eps + b2));
    const T a3 = div_<T>(T(4.0 / 35.0), (eps + b3) * (eps + b3));
    const T sum = a0 + a1 + a2 + a3;
    if (!(sum > T(0)) || !finite_(sum)) flags |= FLAG_NONFINITE;
    return div_<T>(a0 * p0 + a1 * p1 + a2 * p2 + a3 * p3, T(12) * sum);
}

// TENO5 (SF_TENO5.cpp:44-92): C = 1, q = 6, eps = 1e-40, CT = 1e-5.
// keep_mask() is the cut-off decision alone (bit k set = sub-stencil k kept);
// core() is the reconstruction built on it.  `cut` accumulates the number of
// cut sub-stencils.
//
// The sub-stencil polynomials and smoothness indicators are written with
// every rounding fixed (fma where two operations fuse, the _rn intrinsics
// where they must not): left to the compiler, products shared between them
// (2 v2, 3 v2, ...) fuse or not depending on the code around them, so the
// same inputs could round differently in two call sites.
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }

// 6 x the three sub-stencil reconstructions (p_k of the reference).
template <typename T>
__device__ __forceinline__ void teno_polys(const T* v, T& p0, T& p1, T& p2) {
    p0 = fma(T(11), v[2], fma(T(-7), v[1], mul_rn(T(2), v[0])));
    p1 = fma(T(2), v[3], fma(T(5), v[2], -v[1]));
    p2 = add_rn(fma(T(5), v[3], mul_rn(T(2), v[2])), -v[4]);
}

template <typename T>
__device__ __forceinline__ void teno_betas(const T* v, T& b0, T& b1, T& b2) {
    const T t0 = add_rn(fma(T(-2), v[1], v[0]), v[2]), r0 = fma(T(3), v[2], fma(T(-4), v[1], v[0]));
    const T t1 = add_rn(fma(T(-2), v[2], v[1]), v[3]), r1 = add_rn(v[1], -v[3]);
    const T t2 = add_rn(fma(T(-2), v[3], v[2]), v[4]), r2 = add_rn(fma(T(-4), v[3], mul_rn(T(3), v[2])), v[4]);
    const T c13 = T(13.0 / 12.0);
    b0 = fma(c13, mul_rn(t0, t0), mul_rn(T(0.25), mul_rn(r0, r0)));
    b1 = fma(c13, mul_rn(t1, t1), mul_rn(T(0.25), mul_rn(r1, r1)));
    b2 = fma(c13, mul_rn(t2, t2), mul_rn(T(0.25), mul_rn(r2, r2)));
}

template <typename T> struct Teno;

// The smooth-stencil shortcuts below are taken per warp, when every active
// lane's stencils pass: a uniform branch, with no divergent paths to
// reconverge.  A lane whose stencils are smooth but whose warp is not takes
// the cut-off path, which gives it the same bits.
__device__ __forceinline__ bool warp_all(bool p) { return __all_sync(__activemask(), p); }

// d0 p0 + d1 p1 + d2 p2 with its roundings fixed (one product, two fused
// multiply-adds), so a weight set given as constants and the same set chosen
// at run time round alike.
__device__ __forceinline__ double teno_sum64(double d0, double d1, double d2, double p0, double p1, double p2) {
    return fma(d2, p2, fma(d1, p1, d0 * p0));
}

// A smooth sub-stencil triple keeps all three sub-stencils, which the FP64
// cut-off finds only after its division: with tau <= 4 e_min (e_k = b_k +
// 1e-40) every g_k = 1 + tau/e_k lies in [1, 5] up to a few ulps, so G_k >=
// 1 > lim = 1e-5 sum G <= 0.47 and the mask is 7.  b_max <= 1e30 keeps the
// products e0 e1 e2 and the shared reciprocal of two of them finite and
// normal, so the cut-off path raises no non-finite flag either; NaN or
// infinite indicators fail the test.  The weights for mask 7 are then the
// cut-off path's to the bit.
__device__ __forceinline__ bool teno_smooth64(const double (&b)[3], double tau) {
    const double em = fmin(b[0], fmin(b[1], b[2])) + 1e-40;
    return tau <= 4.0 * em && fmax(b[0], fmax(b[1], b[2])) <= 1e30;
}

// FP64 keeps the reference's gamma_k = (1 + tau5/(b_k+eps))^6 and tests
// gamma_k < CT * sum(gamma) (the reference divides; the comparison is the same
// up to rounding at the threshold).
template <> struct Teno<double> {
    static __device__ __forceinline__ int keep_mask(double b0, double b1, double b2, unsigned& flags) {
        const double tau = fabs(b0 - b2);
        // tau/e_k for the three sub-stencils from one reciprocal of the
        // product e0 e1 e2 (>= 1e-120, no underflow in FP64)
        const double e0 = b0 + 1e-40, e1 = b1 + 1e-40, e2 = b2 + 1e-40;
        const double e12 = e1 * e2;
        const double ti = tau / (e0 * e12);
        const double g0 = 1.0 + ti * e12;
        const double g1 = 1.0 + ti * (e0 * e2);
        const double g2 = 1.0 + ti * (e0 * e1);
        const double q0 = g0 * g0 * g0, q1 = g1 * g1 * g1, q2 = g2 * g2 * g2;
        const double G0 = q0 * q0, G1 = q1 * q1, G2 = q2 * q2;
        const double lim = 1e-5 * (G0 + G1 + G2);
        if (!finite_(lim)) flags |= FLAG_NONFINITE;
        return int(!(G0 < lim)) | (int(!(G1 < lim)) << 1) | (int(!(G2 < lim)) << 2);
    }
    static __device__ __forceinline__ double core(const double* v, unsigned& flags, unsigned& cut) {
        double p0, p1, p2, b0, b1, b2;
        teno_polys<double>(v, p0, p1, p2);
        teno_betas<double>(v, b0, b1, b2);
        const double bb[3] = {b0, b1, b2};
        if (warp_all(teno_smooth64(bb, fabs(b0 - b2))))
            return teno_sum64(0.1, 0.6, 0.3, p0, p1, p2) * (1.0 / 6.0);  // mask 7
        const int m = keep_mask(b0, b1, b2, flags);
        cut += 3 - __popc(m);
        if (m == 0) { flags |= FLAG_TENO_CUTOFF; return 0.0; }
        // 1 / (6 * sum of the kept linear weights), by kept set (selects, no
        // indexed local array)
        const double inv6act = m == 7 ? 1.0 / 6.0 : m == 6 ? 1.0 / 5.4 : m == 5 ? 1.0 / 2.4 : m == 4 ? 1.0 / 1.8
                             : m == 3 ? 1.0 / 4.2 : m == 2 ? 1.0 / 3.6 : 1.0 / 0.6;
        const double d0 = (m & 1) ? 0.1 : 0.0, d1 = (m & 2) ? 0.6 : 0.0, d2 = (m & 4) ? 0.3 : 0.0;
        return teno_sum64(d0, d1, d2, p0, p1, p2) * inv6act;
    }
};

// FP32 cut-off, for two independent sub-stencil triples at once (the two
// lanes).  gamma_k = g_k^6 with g_k = 1 + tau/e_k leaves single-precision
// range long before FP64's, so the test is made on the ratios to the largest
// g, which belongs to the smallest e:
//   x_k = g_k / g_max = t + s / e_k,   t = e_min / (e_min + tau),  s = tau t.
// s <= e_min <= e_k, so every x_k lies in (0, 1] (x = 1 for e_min): nothing
// overflows and no 0/0 or 0*inf arises, with no branch.  Keep k iff
// x_k^6 >= CT * sum_j x_j^6 -- the reference's gamma_k / sum gamma >= CT
// divided through by g_max^6.  eps is FLT_MIN: the reference's 1e-40 is
// subnormal in FP32, whose reciprocal leaves the range.  keep[k] = 1 or 0
// (0 for a NaN input, which `bad` reports).
constexpr float TENO32_EPS = 1.17549435e-38f;

__device__ __forceinline__ void teno_keep32x2(float2 b0, float2 b1, float2 b2, float2 (&keep)[3], float2& bad) {
    const float2 e0 = add2(b0, f2(TENO32_EPS)), e1 = add2(b1, f2(TENO32_EPS)), e2 = add2(b2, f2(TENO32_EPS));
    const float2 d02 = sub2(b0, b2);
    const float2 tau = f2(fabsf(d02.x), fabsf(d02.y));
    const float2 em = f2(fminf(e0.x, fminf(e1.x, e2.x)), fminf(e0.y, fminf(e1.y, e2.y)));
    const float2 t = mul2(em, rcp2(add2(em, tau)));
    const float2 s = mul2(tau, t);
    const float2 x0 = fma2(s, rcp2(e0), t), x1 = fma2(s, rcp2(e1), t), x2 = fma2(s, rcp2(e2), t);
    const float2 y0 = mul2(x0, x0), y1 = mul2(x1, x1), y2 = mul2(x2, x2);
    const float2 G0 = mul2(mul2(y0, y0), y0), G1 = mul2(mul2(y1, y1), y1), G2 = mul2(mul2(y2, y2), y2);
    const float2 lim = mul2(f2(1e-5f), add2(add2(G0, G1), G2));
    bad = watch2(bad, lim);  // NaN input (lim <= 3e-5 otherwise)
    keep[0] = f2(ge_one(G0.x, lim.x), ge_one(G0.y, lim.y));
    keep[1] = f2(ge_one(G1.x, lim.x), ge_one(G1.y, lim.y));
    keep[2] = f2(ge_one(G2.x, lim.x), ge_one(G2.y, lim.y));
}

// A smooth stencil pair keeps every sub-stencil, which the cut-off would
// find only after its reciprocals: with tau = |B0 - B2| <= 4 e_min (e_min =
// min B + eps <= 1e30) in both lanes, t = e_min / (e_min + tau) >= 0.2 up to
// a few ulps, every x_k >= t, so G_k >= 6.39e-5 > 2 lim (lim = 1e-5 sum G <=
// 3.0001e-5): teno_keep32x2 would return k = 1 for all three.  The test
// fails for NaN or infinite indicators (they take the cut-off path and its
// non-finite watch), and a pair that passes has finite differences, so the
// weights computed with k = 1 are the cut-off path's to the bit.
__device__ __forceinline__ bool teno_smooth2(const float2 (&B)[3]) {
    const float2 em = add2(f2(fminf(B[0].x, fminf(B[1].x, B[2].x)), fminf(B[0].y, fminf(B[1].y, B[2].y))),
                           f2(TENO32_EPS));
    const float2 d02 = sub2(B[0], B[2]);
    return fabsf(d02.x) <= 4.f * em.x && fabsf(d02.y) <= 4.f * em.y && em.x <= 1e30f && em.y <= 1e30f;
}

template <> struct Teno<float> {
    static __device__ __forceinline__ int keep_mask(float b0, float b1, float b2, unsigned& flags) {
        float2 k[3];
        float2 bad = f2(0.f);
        teno_keep32x2(f2(b0), f2(b1), f2(b2), k, bad);
        flag_bad(bad, flags);
        return int(k[0].x != 0.f) | (int(k[1].x != 0.f) << 1) | (int(k[2].x != 0.f) << 2);
    }
    static __device__ __forceinline__ float core(const float* v, unsigned& flags, unsigned& cut) {
        float p0, p1, p2, b0, b1, b2;
        teno_polys<float>(v, p0, p1, p2);
        teno_betas<float>(v, b0, b1, b2);
        const float2 bb[3] = {f2(b0), f2(b1), f2(b2)};
        if (warp_all(teno_smooth2(bb)))  // mask 7 (teno_smooth2 on both lanes of the broadcast)
            return __fdividef(fmaf(0.3f, p2, fmaf(0.6f, p1, 0.1f * p0)), 6.f * ((0.1f + 0.6f) + 0.3f));
        const int m = keep_mask(b0, b1, b2, flags);
        cut += 3 - __popc(m);
        const float d0 = (m & 1) ? 0.1f : 0.f, d1 = (m & 2) ? 0.6f : 0.f, d2 = (m & 4) ? 0.3f : 0.f;
        const float act = (d0 + d1) + d2;
        if (!(act > 0.f)) { flags |= FLAG_TENO_CUTOFF; return 0.f; }
        return __fdividef(fmaf(d2, p2, fmaf(d1, p1, d0 * p0)), 6.f * act);
    }
};

// FP64 left / right core pairs sharing one division: with x/a and y/b needed,
// r = 1/(a b) gives x b r and y a r.  The WENO5 denominators lie in
// [6e-25, ~1e33] and the TENO5 products e0 e1 e2 in [1e-120, ~1e24] for any
// state the reference accepts, so a b stays inside FP64 range.
__device__ __forceinline__ void weno5_pair64(const double* l, const double* r, double& wl, double& wr,
                                             unsigned& flags) {
    double num[2], den[2];
    const double* v2[2] = {l, r};
#pragma unroll
    for (int side = 0; side < 2; ++side) {
        const double* v = v2[side];
        const double p0 = 2.0 * v[0] - 7.0 * v[1] + 11.0 * v[2];
        const double p1 = -v[1] + 5.0 * v[2] + 2.0 * v[3];
        const double p2 = 2.0 * v[2] + 5.0 * v[3] - v[4];
        const double t0 = v[0] - 2.0 * v[1] + v[2], r0 = v[0] - 4.0 * v[1] + 3.0 * v[2];
        const double t1 = v[1] - 2.0 * v[2] + v[3], r1 = v[1] - v[3];
        const double t2 = v[2] - 2.0 * v[3] + v[4], r2 = 3.0 * v[2] - 4.0 * v[3] + v[4];
        const double c13 = 13.0 / 12.0;
        const double b0 = c13 * (t0 * t0) + 0.25 * (r0 * r0);
        const double b1 = c13 * (t1 * t1) + 0.25 * (r1 * r1);
        const double b2 = c13 * (t2 * t2) + 0.25 * (r2 * r2);
        const double s0 = (1e-6 + b0) * (1e-6 + b0), s1 = (1e-6 + b1) * (1e-6 + b1), s2 = (1e-6 + b2) * (1e-6 + b2);
        const double w0 = 0.1 * (s1 * s2), w1 = 0.6 * (s0 * s2), w2 = 0.3 * (s0 * s1);
        den[side] = 6.0 * (w0 + w1 + w2);
        num[side] = w0 * p0 + w1 * p1 + w2 * p2;
    }
    const double inv = 1.0 / (den[0] * den[1]);
    if (!(inv > 0.0) || !isfinite(inv)) flags |= FLAG_NONFINITE;
    wl = num[0] * den[1] * inv;
    wr = num[1] * den[0] * inv;
}

__device__ __forceinline__ void teno5_pair64(const double* l, const double* r, double& wl, double& wr,
                                             unsigned& flags, unsigned& cut) {
    double b[2][3], p[2][3], e[2][3], tau[2], prod[2];
    const double* v2[2] = {l, r};
#pragma unroll
    for (int side = 0; side < 2; ++side) {
        const double* v = v2[side];
        teno_polys<double>(v, p[side][0], p[side][1], p[side][2]);
        teno_betas<double>(v, b[side][0], b[side][1], b[side][2]);
        tau[side] = fabs(b[side][0] - b[side][2]);
        for (int k = 0; k < 3; ++k) e[side][k] = b[side][k] + 1e-40;
        prod[side] = e[side][0] * (e[side][1] * e[side][2]);
    }
    if (warp_all(teno_smooth64(b[0], tau[0]) && teno_smooth64(b[1], tau[1]))) {
        // every sub-stencil kept on both sides: the m = 7 weights below
        wl = teno_sum64(0.1, 0.6, 0.3, p[0][0], p[0][1], p[0][2]) * (1.0 / 6.0);
        wr = teno_sum64(0.1, 0.6, 0.3, p[1][0], p[1][1], p[1][2]) * (1.0 / 6.0);
        return;
    }
    const double inv = 1.0 / (prod[0] * prod[1]);
    double out[2];
#pragma unroll
    for (int side = 0; side < 2; ++side) {
        // tau / (e0 e1 e2) from the shared reciprocal
        const double ti = tau[side] * prod[1 - side] * inv;
        const double g0 = 1.0 + ti * (e[side][1] * e[side][2]);
        const double g1 = 1.0 + ti * (e[side][0] * e[side][2]);
        const double g2 = 1.0 + ti * (e[side][0] * e[side][1]);
        const double q0 = g0 * g0 * g0, q1 = g1 * g1 * g1, q2 = g2 * g2 * g2;
        const double G0 = q0 * q0, G1 = q1 * q1, G2 = q2 * q2;
        const double lim = 1e-5 * (G0 + G1 + G2);
        if (!isfinite(lim)) flags |= FLAG_NONFINITE;
        const int m = int(!(G0 < lim)) | (int(!(G1 < lim)) << 1) | (int(!(G2 < lim)) << 2);
        cut += 3 - __popc(m);
        if (m == 0) flags |= FLAG_TENO_CUTOFF;
        const double inv6act = m == 7 ? 1.0 / 6.0 : m == 6 ? 1.0 / 5.4 : m == 5 ? 1.0 / 2.4 : m == 4 ? 1.0 / 1.8
                             : m == 3 ? 1.0 / 4.2 : m == 2 ? 1.0 / 3.6 : m == 1 ? 1.0 / 0.6 : 0.0;
        const double d0 = (m & 1) ? 0.1 : 0.0, d1 = (m & 2) ? 0.6 : 0.0, d2 = (m & 4) ? 0.3 : 0.0;
        out[side] = teno_sum64(d0, d1, d2, p[side][0], p[side][1], p[side][2]) * inv6act;
    }
    wl = out[0];
    wr = out[1];
}

template <int SCHEME, typename T>
__device__ __forceinline__ T recon_core(const T* v, unsigned& flags, unsigned& cut) {
    if constexpr (SCHEME == WENO5) return weno5_core<T>(v, flags);
    else if constexpr (SCHEME == TENO5) return Teno<T>::core(v, flags, cut);
    else if constexpr (SCHEME == WENO3) return weno3_core<T>(v, flags);
    else return weno7_core<T>(v, flags);
}

// ---------------------------------------------------------------------------
// Face fluxes (per unit area, unit normal = axis AX).
// ---------------------------------------------------------------------------

// Rusanov with both sides closed by the perfect-gas EOS
// (RusanovEOS::faceFlux, SF_rusanovEOS.cpp:47-77; close() of
// SF_singleFluidStateModel.cpp:49-73).
template <int AX, typename T>
__device__ __forceinline__ void rusanov(const T qL[5], const T qR[5], T gamma, T F[5], unsigned& flags) {
    constexpr int N = AxisBasis<AX>::N;
    const T iL = rcp<T>(qL[0]), iR = rcp<T>(qR[0]);
    const T uL[3] = {qL[1] * iL, qL[2] * iL, qL[3] * iL};
    const T uR[3] = {qR[1] * iR, qR[2] * iR, qR[3] * iR};
    const T kL = T(0.5) * qL[0] * (uL[0] * uL[0] + uL[1] * uL[1] + uL[2] * uL[2]);
    const T kR = T(0.5) * qR[0] * (uR[0] * uR[0] + uR[1] * uR[1] + uR[2] * uR[2]);
    const T pL = (gamma - T(1)) * (qL[4] - kL);
    const T pR = (gamma - T(1)) * (qR[4] - kR);
    if (!(qL[0] > T(0)) || !(qR[0] > T(0))) flags |= FLAG_DENSITY;
    if (!(pL > T(0)) || !(pR > T(0))) flags |= FLAG_PRESSURE;
    const T cL = sqrt_<T>(gamma * pL * iL), cR = sqrt_<T>(gamma * pR * iR);
    const T unL = uL[N - 1], unR = uR[N - 1];
    const T lam = fmax(fabs(unL) + cL, fabs(unR) + cR);
    const T hl = T(0.5) * lam;
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        T fl = qL[v] * unL, fr = qR[v] * unR;
        if (v == N) { fl += pL; fr += pR; }
        if (v == 4) { fl += pL * unL; fr += pR * unR; }
        F[v] = T(0.5) * (fl + fr) - hl * (qR[v] - qL[v]);
    }
}

// Roe with the Harten entropy fix (RoeFlux::flux, SF_roe.cpp:20-111).
template <int AX, typename T>
__device__ __forceinline__ void roe(const T qL[5], const T qR[5], T gamma, T F[5], unsigned& flags) {
    constexpr int N = AxisBasis<AX>::N;
    const T gm1 = gamma - T(1);
    const T iL = rcp<T>(qL[0]), iR = rcp<T>(qR[0]);
    const T keL = T(0.5) * (qL[1] * qL[1] + qL[2] * qL[2] + qL[3] * qL[3]) * iL;
    const T keR = T(0.5) * (qR[1] * qR[1] + qR[2] * qR[2] + qR[3] * qR[3]) * iR;
    const T pL = gm1 * (qL[4] - keL), pR = gm1 * (qR[4] - keR);
    if (!(qL[0] > T(0)) || !(qR[0] > T(0))) flags |= FLAG_DENSITY;
    if (!(pL > T(0)) || !(pR > T(0))) flags |= FLAG_PRESSURE;
    const T uL[3] = {qL[1] * iL, qL[2] * iL, qL[3] * iL};
    const T uR[3] = {qR[1] * iR, qR[2] * iR, qR[3] * iR};
    const T hL = (qL[4] + pL) * iL, hR = (qR[4] + pR) * iR;
    const T sL = sqrt_<T>(qL[0]), sR = sqrt_<T>(qR[0]);
    const T iS = rcp<T>(sL + sR);
    const T ur = (sL * uL[0] + sR * uR[0]) * iS;
    const T vr = (sL * uL[1] + sR * uR[1]) * iS;
    const T wr = (sL * uL[2] + sR * uR[2]) * iS;
    const T hr = (sL * hL + sR * hR) * iS;
    const T q2 = ur * ur + vr * vr + wr * wr;
    const T a2 = gm1 * (hr - T(0.5) * q2);
    if (!(a2 > T(0)) || !finite_(a2)) flags |= FLAG_ROE_SOUND;
    const T rr = sL * sR;
    T qr[5] = {rr, rr * ur, rr * vr, rr * wr, rr * (T(0.5) * q2 + div_<T>(a2, gm1))};
    Eigen<T> e;
    eigen_at<AX, T>(qr, gamma, e);
    const T a = sqrt_<T>(a2);
    const T un = (N == 1 ? ur : (N == 2 ? vr : wr));
    const T lam[5] = {un, un, un, un + a, un - a};
    const T delta = T(0.1) * a;
    T dq[5], alpha[5], s[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) dq[v] = qR[v] - qL[v];
    to_characteristic<AX, T>(e, dq, alpha);
    // the reference's wave order is (u_n, u_n, u_n, u_n + a, u_n - a) against
    // columns (w0, w1, w2, w3, w4) of R = (entropy, shear l, shear m, u-c, u+c)
#pragma unroll
    for (int m = 0; m < 5; ++m) {
        const T val = fabs(lam[m]);
        const T ab = val < T(2) * delta ? T(0.5) * (val * val * rcp<T>(T(2) * delta) + delta) : val;
        s[m] = ab * alpha[m];
    }
    T diss[5];
    from_characteristic<AX, T>(e, s, diss);
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        T fl = qL[v] * uL[N - 1], fr = qR[v] * uR[N - 1];
        if (v == N) { fl += pL; fr += pR; }
        if (v == 4) { fl += pL * uL[N - 1]; fr += pR * uR[N - 1]; }
        F[v] = T(0.5) * (fl + fr - diss[v]);
    }
}

// One characteristic face flux (characteristicWENOFaceFlux, SF_WENO.h:184-245)
// from NST conservative points st[0..NST-1] (face between NST/2-1 and NST/2).
// In FP32 the reconstruction runs on deviations from the face average q-bar
// (computed in FP64): the projections are linear and the WENO/TENO cores are
// invariant to adding a constant, so the result is the same mathematics while
// single precision only has to resolve the variation across the stencil.
// Pressure of a conserved state as Numerics::pressure (SF_utility.h:24-29),
// with the validation flags of requirePhysicalState.
template <typename T>
__device__ __forceinline__ T state_pressure(const T q[5], T gamma, T inv_rho, unsigned& flags) {
    const T ke = T(0.5) * (q[1] * q[1] + q[2] * q[2] + q[3] * q[3]) * inv_rho;
    const T p = (gamma - T(1)) * (q[4] - ke);
    if (!(q[0] > T(0))) flags |= FLAG_DENSITY;
    if (!(p > T(0))) flags |= FLAG_PRESSURE;
    return p;
}

// Steger-Warming split of one state (Riemann::splitStegerWarming,
// SF_riemann.cpp:15-67), the positive (POS) or negative part, for the unit
// normal e_AX: eigenvalues u_n, u_n +- a split with the entropy fix of width
// 2 eps, eps = 0.01.
template <int AX, bool POS, typename T>
__device__ __forceinline__ void steger_part(const T q[5], T gamma, T f[5], unsigned& flags) {
    constexpr int N = AxisBasis<AX>::N;
    const T r = q[0];
    const T inv = rcp<T>(r);
    const T p = state_pressure<T>(q, gamma, inv, flags);
    const T vel[3] = {q[1] * inv, q[2] * inv, q[3] * inv};
    const T q2 = vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2];
    const T a = sqrt_<T>(gamma * p * inv);
    const T un = vel[N - 1];
    const T eps = T(0.01);
    auto part = [&](T lam) {
        if (fabs(lam) < T(2) * eps) {
            const T lp = T(0.5) * (lam * lam / (T(4) * eps) + lam + eps);
            return POS ? lp : lam - lp;
        }
        return POS ? T(0.5) * (lam + fabs(lam)) : T(0.5) * (lam - fabs(lam));
    };
    const T l0 = part(un), l3 = part(un + a), l4 = part(un - a);
    const T common = r / (T(2) * gamma);
    const T W1 = T(2) * (gamma - T(1)) * l0 + l3 + l4;
    const T W2 = l3 - l4;
    const T W3 = l3 + l4;
    f[0] = common * W1;
#pragma unroll
    for (int k = 0; k < 3; ++k) f[1 + k] = common * (vel[k] * W1 + (k == N - 1 ? a * W2 : T(0)));
    f[4] = common * (T(0.5) * q2 * W1 + a * un * W2 + (a * a / (gamma - T(1))) * W3);
}

// StegerWarmingFlux::flux (Flux/SF_sw.cpp:22-28): F+(qL) + F-(qR).
template <int AX, typename T>
__device__ __forceinline__ void steger(const T qL[5], const T qR[5], T gamma, T F[5], unsigned& flags) {
    T fp[5], fm[5];
    steger_part<AX, true, T>(qL, gamma, fp, flags);
    steger_part<AX, false, T>(qR, gamma, fm, flags);
#pragma unroll
    for (int v = 0; v < 5; ++v) F[v] = fp[v] + fm[v];
}

// Lax-Friedrichs split (Riemann::splitLaxFriedrichs, SF_riemann.cpp:125-152)
// and LaxFriedrichsFlux::flux (Flux/SF_lxF.cpp): (F(qL) + lam_L qL)/2 +
// (F(qR) - lam_R qR)/2 with each state's own lam = |u_n| + a.
template <int AX, typename T>
__device__ __forceinline__ void laxf_part(const T q[5], T gamma, T sign, T f[5], unsigned& flags) {
    constexpr int N = AxisBasis<AX>::N;
    const T inv = rcp<T>(q[0]);
    const T p = state_pressure<T>(q, gamma, inv, flags);
    const T un = q[N] * inv;
    const T lam = fabs(un) + sqrt_<T>(gamma * p * inv);
    T Fp[5];
    Fp[0] = q[0] * un;
#pragma unroll
    for (int k = 0; k < 3; ++k) Fp[1 + k] = q[1 + k] * un + (k == N - 1 ? p : T(0));
    Fp[4] = (q[4] + p) * un;
#pragma unroll
    for (int v = 0; v < 5; ++v) f[v] = T(0.5) * (Fp[v] + sign * lam * q[v]);
}

template <int AX, typename T>
__device__ __forceinline__ void laxf(const T qL[5], const T qR[5], T gamma, T F[5], unsigned& flags) {
    T fp[5], fm[5];
    laxf_part<AX, T>(qL, gamma, T(1), fp, flags);
    laxf_part<AX, T>(qR, gamma, T(-1), fm, flags);
#pragma unroll
    for (int v = 0; v < 5; ++v) F[v] = fp[v] + fm[v];
}

// physicalEulerFlux (Flux/SF_face.h:112-127) along e_AX.
template <int AX, typename T>
__device__ __forceinline__ void euler_flux(const T q[5], T gamma, T f[5], unsigned& flags) {
    constexpr int N = AxisBasis<AX>::N;
    const T rho = q[0];
    const T inv = rcp<T>(rho);
    const T p = state_pressure<T>(q, gamma, inv, flags);
    const T vel[3] = {q[1] * inv, q[2] * inv, q[3] * inv};
    const T un = vel[N - 1];
    f[0] = rho * un;
#pragma unroll
    for (int k = 0; k < 3; ++k) f[1 + k] = rho * vel[k] * un + (k == N - 1 ? p : T(0));
    f[4] = (q[4] + p) * un;
}

// LaxWendroffFlux::flux (Flux/SF_lw.cpp:17-40): the physical flux of the
// Richtmyer half-step state (qL + qR)/2 - lam/2 (F(qR) - F(qL)), lam = dt / h.
template <int AX, typename T>
__device__ __forceinline__ void laxw(const T qL[5], const T qR[5], T gamma, T lam, T F[5], unsigned& flags) {
    T fL[5], fR[5], qh[5];
    euler_flux<AX, T>(qL, gamma, fL, flags);
    euler_flux<AX, T>(qR, gamma, fR, flags);
#pragma unroll
    for (int v = 0; v < 5; ++v) qh[v] = T(0.5) * (qL[v] + qR[v]) - T(0.5) * lam * (fR[v] - fL[v]);
    euler_flux<AX, T>(qh, gamma, F, flags);
}

// `lam` = dt / h along AX, used by the Lax-Wendroff flux only.
template <int AX, int SCHEME, int FLUX, typename T>
__device__ __forceinline__ void face_flux(const double (&st)[SchemeInfo<SCHEME>::NST][5], T gamma, T F[5],
                                          unsigned& flags, unsigned& cut, T lam = T(0)) {
    constexpr int NST = SchemeInfo<SCHEME>::NST;
    constexpr int W = SchemeInfo<SCHEME>::W;
    constexpr int CL = NST / 2 - 1;
    constexpr bool DEV = sizeof(T) < sizeof(double);
    double qbar64[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) qbar64[v] = 0.5 * (st[CL][v] + st[CL + 1][v]);
    T qbar[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) qbar[v] = T(qbar64[v]);
    Eigen<T> e;
    if (!eigen_at<AX, T>(qbar, gamma, e)) flags |= FLAG_PRESSURE;
    T ch[NST][5];
#pragma unroll
    for (int s = 0; s < NST; ++s) {
        T d[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) d[v] = DEV ? T(st[s][v] - qbar64[v]) : T(st[s][v]);
        to_characteristic<AX, T>(e, d, ch[s]);
    }
    T wl[5], wr[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        T sl[W], sr[W];
#pragma unroll
        for (int s = 0; s < W; ++s) {
            sl[s] = ch[s][v];
            sr[s] = ch[NST - 1 - s][v];
        }
        if constexpr (sizeof(T) == sizeof(double) && SCHEME == WENO5) {
            weno5_pair64(sl, sr, wl[v], wr[v], flags);
        } else if constexpr (sizeof(T) == sizeof(double) && SCHEME == TENO5) {
            teno5_pair64(sl, sr, wl[v], wr[v], flags, cut);
        } else {
            wl[v] = recon_core<SCHEME, T>(sl, flags, cut);
            wr[v] = recon_core<SCHEME, T>(sr, flags, cut);
        }
    }
    T dl[5], dr[5], ql[5], qr[5];
    from_characteristic<AX, T>(e, wl, dl);
    from_characteristic<AX, T>(e, wr, dr);
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        ql[v] = DEV ? T(qbar64[v] + double(dl[v])) : dl[v];
        qr[v] = DEV ? T(qbar64[v] + double(dr[v])) : dr[v];
    }
    if constexpr (FLUX == RUSANOV) rusanov<AX, T>(ql, qr, gamma, F, flags);
    else if constexpr (FLUX == ROE) roe<AX, T>(ql, qr, gamma, F, flags);
    else if constexpr (FLUX == STEGER) steger<AX, T>(ql, qr, gamma, F, flags);
    else if constexpr (FLUX == LAXF) laxf<AX, T>(ql, qr, gamma, F, flags);
    else laxw<AX, T>(ql, qr, gamma, lam, F, flags);
#pragma unroll
    for (int v = 0; v < 5; ++v)
        if (!finite_(F[v])) flags |= FLAG_NONFINITE;
}

// ---------------------------------------------------------------------------
// Paired FP32 cores.  The left- and right-biased reconstructions of a face
// are the same operations on mirrored stencils, so they run as the two
// halves of a float2.
// ---------------------------------------------------------------------------

// The 5-point stencil in first differences D_i = v_{i+1} - v_i (both lanes):
//   t0 = D1 - D0, t1 = D2 - D1, t2 = D3 - D2          (second differences)
//   r0 = 3 D1 - D0 = t0 + 2 D1, r1 = D1 + D2, r2 = D3 - 3 D2 = t2 - 2 D2
//   B_k = 12 b_k = 13 t_k^2 + 3 r_k^2
//   p_k - 6 v2 = q_k:  q0 = 5 D1 - 2 D0 = 2 t0 + 3 D1, q1 = D1 + 2 D2, q2 = 4 D2 - D3 = D2 - r2
// (r1 is the reference's v1 - v3 up to sign, which the square removes), so a
// reconstruction sum w_k p_k / (6 sum w_k) is v2 + sum w_k q_k / (6 sum w_k).
// The indicators are returned as B_k / 3 = 4 b_k = 13/3 t_k^2 + r_k^2 (one
// multiply fewer than 12 b_k) and the epsilons are scaled with them, which
// leaves every weight unchanged; only differences of the stencil are rounded.
__device__ __forceinline__ void stencil5x2(const float2* v, float2 (&B)[3], float2 (&q)[3]) {
    const float2 D0 = sub2(v[1], v[0]), D1 = sub2(v[2], v[1]), D2 = sub2(v[3], v[2]), D3 = sub2(v[4], v[3]);
    const float2 t0 = sub2(D1, D0), t1 = sub2(D2, D1), t2 = sub2(D3, D2);
    const float2 r0 = fma2(f2(2.f), D1, t0), r1 = add2(D1, D2), r2 = fma2(f2(-2.f), D2, t2);
    const float2 c = f2(13.f / 3.f);
    B[0] = fma2(mul2(c, t0), t0, mul2(r0, r0));
    B[1] = fma2(mul2(c, t1), t1, mul2(r1, r1));
    B[2] = fma2(mul2(c, t2), t2, mul2(r2, r2));
    q[0] = fma2(f2(2.f), t0, mul2(f2(3.f), D1));
    q[1] = fma2(f2(2.f), D2, D1);
    q[2] = sub2(D2, r2);
}

// WENO5-JS on a (left, right) stencil pair; same folding as weno5_core.
__device__ __forceinline__ float2 weno5_core2(const float2* v, float2& bad) {
    float2 B[3], q[3];
    stencil5x2(v, B, q);
    const float2 eps = f2(4.f * 1e-6f);  // the reference's 1e-6 on B_k / 3 = 4 b_k
    const float2 e0 = add2(eps, B[0]), e1 = add2(eps, B[1]), e2 = add2(eps, B[2]);
    const float2 s0 = mul2(e0, e0), s1 = mul2(e1, e1), s2 = mul2(e2, e2);
    const float2 w0 = mul2(f2(0.1f), mul2(s1, s2));
    const float2 w1 = mul2(f2(0.6f), mul2(s0, s2));
    const float2 w2 = mul2(f2(0.3f), mul2(s0, s1));
    const float2 den = mul2(f2(6.f), add2(add2(w0, w1), w2));
    const float2 num = fma2(w0, q[0], fma2(w1, q[1], mul2(w2, q[2])));
    bad = watch2(bad, den);  // den >= 6 eps^4 > 0 unless an input was not finite
    return fma2(num, rcp2(den), v[2]);
}

// TENO5 on a (left, right) stencil pair, all of it paired: polynomials,
// smoothness indicators, the cut-off (teno_keep32x2) and the weights.  With
// `count` (a launch-uniform switch: the cut-off accounting of
// sfg_set_counting), `kept` accumulates the kept sub-stencils of each lane.
// TENO5 weights from the keep flags k (1 or 0 per lane): the kept linear
// weights, renormalised.  No all-cut check: the sub-stencil with x = 1
// always passes (G ~ 1 > lim <= 3e-5, and a NaN lim fails every '<'), so
// act >= 0.6.
__device__ __forceinline__ float2 teno5_weights2(const float2 (&k)[3], const float2 (&q)[3], float2 v2) {
    const float2 d0 = mul2(f2(0.1f), k[0]), d1 = mul2(f2(0.6f), k[1]), d2 = mul2(f2(0.3f), k[2]);
    const float2 act = fma2(f2(6.f), d0, fma2(f2(6.f), d1, mul2(f2(6.f), d2)));
    const float2 num = fma2(d0, q[0], fma2(d1, q[1], mul2(d2, q[2])));
    return fma2(num, rcp2(act), v2);
}

__device__ __forceinline__ float2 teno5_core2(const float2* v, float2& bad, bool count, float2& kept) {
    float2 B[3], q[3], k[3];
    stencil5x2(v, B, q);
    if (warp_all(teno_smooth2(B))) {
        const float2 all[3] = {f2(1.f), f2(1.f), f2(1.f)};
        if (count) kept = add2(kept, f2(3.f));
        return teno5_weights2(all, q, v[2]);
    }
    teno_keep32x2(B[0], B[1], B[2], k, bad);
    if (count) kept = add2(kept, add2(add2(k[0], k[1]), k[2]));
    return teno5_weights2(k, q, v[2]);
}

// The eigen-structure as lane pairs, signs folded in, built once per face.
// The tangential characteristic variables are taken with the raw Cartesian
// components, w_t = m_t - u_t rho: the reference's signed tangents (+-e_t)
// only negate w_t, and negation commutes exactly with the projection, every
// reconstruction core (linear polynomials, squared indicators) and the
// back-projection, so the face states are bit-identical.
struct Eig2 {
    float2 u[3], nu[3];  // velocity, negated velocity
    float2 h, H, c, nb1, b2, x1, nx1;
};

__device__ __forceinline__ Eig2 eig2(const Eigen<float>& e) {
    Eig2 p;
    p.u[0] = f2(e.u), p.u[1] = f2(e.v), p.u[2] = f2(e.w);
    p.nu[0] = f2(-e.u), p.nu[1] = f2(-e.v), p.nu[2] = f2(-e.w);
    p.h = f2(e.h), p.H = f2(e.H), p.c = f2(e.c);
    p.nb1 = f2(-e.b1), p.b2 = f2(e.b2), p.x1 = f2(e.x1), p.nx1 = f2(-e.x1);
    return p;
}

// Characteristic projection of a pair of points:
//   -A = E + h rho - u.m,  -B = m_n - u_n rho,
//   w0 = rho - b1 (-A),  w3 = -x1 (-B) + b2 (-A),  w4 = x1 (-B) + b2 (-A).
template <int AX>
__device__ __forceinline__ void to_characteristic2(const Eig2& e, const float2 q[5], float2 w[5]) {
    using B = AxisBasis<AX>;
    const float2 nA = fma2(e.nu[0], q[1], fma2(e.nu[1], q[2], fma2(e.nu[2], q[3], fma2(e.h, q[0], q[4]))));
    const float2 nB = fma2(e.nu[B::N - 1], q[0], q[B::N]);
    const float2 b2nA = mul2(e.b2, nA);
    w[0] = fma2(e.nb1, nA, q[0]);
    w[1] = fma2(e.nu[B::L - 1], q[0], q[B::L]);
    w[2] = fma2(e.nu[B::M - 1], q[0], q[B::M]);
    w[3] = fma2(e.nx1, nB, b2nA);
    w[4] = fma2(e.x1, nB, b2nA);
}

template <int AX>
__device__ __forceinline__ void from_characteristic2(const Eig2& e, const float2 w[5], float2 q[5]) {
    using B = AxisBasis<AX>;
    const float2 S = add2(add2(w[0], w[3]), w[4]);
    const float2 cD = mul2(e.c, sub2(w[4], w[3]));
    q[0] = S;
    q[B::N] = fma2(e.u[B::N - 1], S, cD);
    q[B::L] = fma2(e.u[B::L - 1], S, w[1]);
    q[B::M] = fma2(e.u[B::M - 1], S, w[2]);
    q[4] = fma2(e.h, w[0], fma2(e.u[B::L - 1], w[1], fma2(e.u[B::M - 1], w[2],
                fma2(e.H, add2(w[3], w[4]), mul2(e.u[B::N - 1], cD)))));
}

// Reference state of a tile in FP32 with its velocity and pressure.
struct Ref32 {
    float q[5];
    float u[3];
    float p;
};

__device__ __forceinline__ Ref32 make_ref32(const double (&qref)[5], double gamma) {
    Ref32 r;
    const double inv = 1.0 / qref[0];
    const double u0 = qref[1] * inv, u1 = qref[2] * inv, u2 = qref[3] * inv;
    const double p = (gamma - 1.0) * (qref[4] - 0.5 * (qref[1] * u0 + qref[2] * u1 + qref[3] * u2));
    for (int v = 0; v < 5; ++v) r.q[v] = float(qref[v]);
    r.u[0] = float(u0);
    r.u[1] = float(u1);
    r.u[2] = float(u2);
    r.p = float(p);
    return r;
}

// Physical Euler flux along axis AX of q = q_ref + d, returned as the
// deviation F(q) - F(q_ref), in algebra that never forms a small difference
// of large terms:
//   du = (d_m - u_ref d_rho) / rho,  u = u_ref + du
//   d(m.u) = m_ref.du + d_m.u,  dp = (gamma - 1)(d_E - d(m.u)/2)
//   dF_rho = d_m_n,  dF_m = m_ref du_n + d_m u_n + dp e_n,
//   dF_E = (E_ref + p_ref) du_n + (d_E + dp) u_n.
// Also gives u_n and the sound speed of q.
template <int AX>
__device__ __forceinline__ void phys_flux_dev(const Ref32& r, const float d[5], float gamma, float F[5], float& un,
                                              float& c, float& p_out, unsigned& flags) {
    constexpr int N = AxisBasis<AX>::N;
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
    const float dun = du[N - 1];
    un = u[N - 1];
    F[0] = d[N];
#pragma unroll
    for (int k = 0; k < 3; ++k) F[1 + k] = r.q[1 + k] * dun + d[1 + k] * un + (k == N - 1 ? dp : 0.f);
    F[4] = (r.q[4] + r.p) * dun + (d[4] + dp) * un;
    c = sqrtf(gamma * p * irho);
    p_out = p;
}

// Rusanov flux deviation F-hat(q_ref + dL, q_ref + dR) - F(q_ref): the
// central part from phys_flux_dev, the dissipation from dR - dL.
template <int AX>
__device__ __forceinline__ void rusanov_dev(const Ref32& r, const float dL[5], const float dR[5], float gamma,
                                            float F[5], unsigned& flags, float scale = 1.f) {
    float fL[5], fR[5], unL, unR, cL, cR, pL, pR;
    phys_flux_dev<AX>(r, dL, gamma, fL, unL, cL, pL, flags);
    phys_flux_dev<AX>(r, dR, gamma, fR, unR, cR, pR, flags);
    const float hl = 0.5f * fmaxf(fabsf(unL) + cL, fabsf(unR) + cR);
#pragma unroll
    for (int v = 0; v < 5; ++v) F[v] = (0.5f * (fL[v] + fR[v]) - hl * (dR[v] - dL[v])) * scale;
}

// Roe flux deviation: Roe average and eigen-structure from the absolute
// states, jump dR - dL, central part from phys_flux_dev.
template <int AX>
__device__ __forceinline__ void roe_dev(const Ref32& r, const float dL[5], const float dR[5], float gamma, float F[5],
                                        unsigned& flags, float scale = 1.f) {
    constexpr int N = AxisBasis<AX>::N;
    float qL[5], qR[5], fL[5], fR[5], unL, unR, cL, cR, pL, pR;
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        qL[v] = r.q[v] + dL[v];
        qR[v] = r.q[v] + dR[v];
    }
    phys_flux_dev<AX>(r, dL, gamma, fL, unL, cL, pL, flags);
    phys_flux_dev<AX>(r, dR, gamma, fR, unR, cR, pR, flags);
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
    float qr[5] = {rr, rr * ur, rr * vr, rr * wr, rr * (0.5f * q2 + __fdividef(a2, gm1))};
    Eigen<float> e;
    eigen_at<AX, float>(qr, gamma, e);
    const float a = sqrtf(a2);
    const float un = (N == 1 ? ur : (N == 2 ? vr : wr));
    const float lam[5] = {un, un, un, un + a, un - a};
    const float delta = 0.1f * a;
    float dq[5], alpha[5], s[5], diss[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) dq[v] = dR[v] - dL[v];
    to_characteristic<AX, float>(e, dq, alpha);
#pragma unroll
    for (int m = 0; m < 5; ++m) {
        const float val = fabsf(lam[m]);
        const float ab = val < 2.f * delta ? 0.5f * (val * val * rcp_approx(2.f * delta) + delta) : val;
        s[m] = ab * alpha[m];
    }
    from_characteristic<AX, float>(e, s, diss);
#pragma unroll
    for (int v = 0; v < 5; ++v) F[v] = (fL[v] + fR[v] - diss[v]) * (0.5f * scale);
}

// phys_flux_dev for the (left, right) pair of face states.  Reciprocal and
// square root use the SFU approximations (rcp, rsqrt): their ~1 ulp error
// sits in front of quantities that are already deviations.
template <int AX>
__device__ __forceinline__ void phys_flux_dev2(const Ref32& r, const float2 d[5], float gamma, float2 F[5], float2& un,
                                               float2& c, unsigned& flags) {
    constexpr int N = AxisBasis<AX>::N;
    const float2 rho = add2(f2(r.q[0]), d[0]);
    const float2 irho = rcp2(rho);
    float2 du[3], u[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        du[k] = mul2(fma2(f2(-r.u[k]), d[0], d[1 + k]), irho);
        u[k] = add2(f2(r.u[k]), du[k]);
    }
    const float2 dmu = fma2(f2(r.q[1]), du[0], fma2(f2(r.q[2]), du[1], fma2(f2(r.q[3]), du[2],
                       fma2(d[1], u[0], fma2(d[2], u[1], mul2(d[3], u[2]))))));
    const float2 dp = mul2(f2(gamma - 1.f), fma2(f2(-0.5f), dmu, d[4]));
    const float2 p = add2(f2(r.p), dp);
    if (!(rho.x > 0.f) || !(rho.y > 0.f)) flags |= FLAG_DENSITY;
    if (!(p.x > 0.f) || !(p.y > 0.f)) flags |= FLAG_PRESSURE;
    const float2 dun = du[N - 1];
    un = u[N - 1];
    F[0] = d[N];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        F[1 + k] = fma2(f2(r.q[1 + k]), dun, mul2(d[1 + k], un));
        if (k == N - 1) F[1 + k] = add2(F[1 + k], dp);
    }
    F[4] = fma2(f2(r.q[4] + r.p), dun, mul2(add2(d[4], dp), un));
    const float2 x = mul2(mul2(f2(gamma), p), irho);
    c = f2(x.x * rsqrtf(x.x), x.y * rsqrtf(x.y));
}

template <int AX>
__device__ __forceinline__ void rusanov_dev2(const Ref32& r, const float2 d[5], float gamma, float F[5],
                                             unsigned& flags, float scale = 1.f) {
    float2 f[5], un, c;
    phys_flux_dev2<AX>(r, d, gamma, f, un, c, flags);
    // F = (f_L + f_R)/2 - lam/2 (d_R - d_L) = ((f_L + lam d_L) + (f_R - lam d_R)) / 2
    const float lam = fmaxf(fabsf(un.x) + c.x, fabsf(un.y) + c.y);
    const float2 lr = f2(lam, -lam);
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        const float2 g = fma2(lr, d[v], f[v]);
        F[v] = (g.x + g.y) * (0.5f * scale);
    }
}

// face_flux_dev32 with the left / right work paired in float2 (WENO5, TENO5).
template <int AX, int SCHEME, int FLUX>
__device__ __forceinline__ void face_flux_dev32x2(const float (&d)[6][5], const Ref32& ref, float gamma, float F[5],
                                                  unsigned& flags, unsigned& cut, bool count, float scale) {
    float dbar[5], qbar[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        dbar[v] = 0.5f * (d[2][v] + d[3][v]);
        qbar[v] = ref.q[v] + dbar[v];
    }
    Eigen<float> es;
    if (!eigen_at<AX, float>(qbar, gamma, es)) flags |= FLAG_PRESSURE;
    const Eig2 e = eig2(es);
    // point pairs (k, 5-k): P[k][v] = (c_k, c_{5-k}) of component v
    float2 P[3][5];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float2 x[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) x[v] = sub2(f2(d[k][v], d[5 - k][v]), f2(dbar[v]));
        to_characteristic2<AX>(e, x, P[k]);
    }
    float2 w[5];
    float2 kept = f2(0.f), bad = f2(0.f);
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        // left stencil c0..c4 and right stencil c5..c1 as one paired stencil
        const float2 st[5] = {P[0][v], P[1][v], P[2][v], swap2(P[2][v]), swap2(P[1][v])};
        if constexpr (SCHEME == TENO5) w[v] = teno5_core2(st, bad, count, kept);
        else w[v] = weno5_core2(st, bad);
    }
    flag_bad(bad, flags);
    if constexpr (SCHEME == TENO5) {
        if (count) cut += 30u - unsigned(kept.x + kept.y);
    }
    float2 dq[5], x2[5];
    from_characteristic2<AX>(e, w, dq);
#pragma unroll
    for (int v = 0; v < 5; ++v) x2[v] = add2(f2(dbar[v]), dq[v]);  // (left, right) deviations from q_ref
    if constexpr (FLUX == RUSANOV) {
        rusanov_dev2<AX>(ref, x2, gamma, F, flags, scale);
    } else {
        float xl[5], xr[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            xl[v] = x2[v].x;
            xr[v] = x2[v].y;
        }
        roe_dev<AX>(ref, xl, xr, gamma, F, flags, scale);
    }
}

// FP32 face flux from a stencil held as FP32 deviations d_s = q_s - q_ref
// from a reference state shared by a whole stage launch (q_ref is FP64 in
// HBM; only the deviations are rounded to FP32, once per node when a tile is
// staged).  Same mathematics as face_flux: q-bar = q_ref + (d_CL + d_CL+1)/2,
// the projection and reconstruction act on d_s - d-bar.  Returns the flux as
// a deviation from F(q_ref) (rusanov_dev / roe_dev): the reference flux
// cancels exactly in every difference dF, so FP32 rounding scales with the
// distance from the reference state, not with |F|.
// `count`: the launch's TENO5 cut-off accounting is on (sfg_set_counting);
// `cut` then receives the cut sub-stencils of the face.  `scale` multiplies
// the flux (a face area): folded into the flux's closing factor 1/2, which
// is exact, so F * scale rounds as one multiply after the flux would.
template <int AX, int SCHEME, int FLUX>
__device__ __forceinline__ void face_flux_dev32(const float (&d)[SchemeInfo<SCHEME>::NST][5], const Ref32& ref,
                                                float gamma, float F[5], unsigned& flags, unsigned& cut,
                                                bool count = true, float scale = 1.f) {
    if constexpr (SCHEME == WENO5 || SCHEME == TENO5) {
        face_flux_dev32x2<AX, SCHEME, FLUX>(d, ref, gamma, F, flags, cut, count, scale);
        return;
    }
    const float (&qref)[5] = ref.q;
    constexpr int NST = SchemeInfo<SCHEME>::NST;
    constexpr int W = SchemeInfo<SCHEME>::W;
    constexpr int CL = NST / 2 - 1;
    float dbar[5], qbar[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        dbar[v] = 0.5f * (d[CL][v] + d[CL + 1][v]);
        qbar[v] = qref[v] + dbar[v];
    }
    Eigen<float> e;
    if (!eigen_at<AX, float>(qbar, gamma, e)) flags |= FLAG_PRESSURE;
    float ch[NST][5];
#pragma unroll
    for (int s = 0; s < NST; ++s) {
        float dd[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) dd[v] = d[s][v] - dbar[v];
        to_characteristic<AX, float>(e, dd, ch[s]);
    }
    float wl[5], wr[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        float sl[W], sr[W];
#pragma unroll
        for (int s = 0; s < W; ++s) {
            sl[s] = ch[s][v];
            sr[s] = ch[NST - 1 - s][v];
        }
        wl[v] = recon_core<SCHEME, float>(sl, flags, cut);
        wr[v] = recon_core<SCHEME, float>(sr, flags, cut);
    }
    float dl[5], dr[5], xl[5], xr[5];
    from_characteristic<AX, float>(e, wl, dl);
    from_characteristic<AX, float>(e, wr, dr);
#pragma unroll
    for (int v = 0; v < 5; ++v) {  // face states as deviations from q_ref
        xl[v] = dbar[v] + dl[v];
        xr[v] = dbar[v] + dr[v];
    }
    if constexpr (FLUX == RUSANOV) rusanov_dev<AX>(ref, xl, xr, gamma, F, flags, scale);
    else roe_dev<AX>(ref, xl, xr, gamma, F, flags, scale);
}

}  // namespace sfg
