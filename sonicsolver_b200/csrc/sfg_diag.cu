// sfg_diag.cu -- measurement aids: the FMA throughput of the GPU (the FP64 /
// FP32 roof of the flux kernels) and per-sweep timing on the solver stream.
#include "../../include/sonicsolver_b200.h"
#include "sfg_internal.h"
#include "sfg_math.cuh"
#include "sfg_stage.cuh"

#include <cstdio>
#include <string>

namespace sfg {

// TENO5 cut-off decisions of the same stencils evaluated in FP64 (the plain
// path) and in FP32 (the FP32-flux path's arithmetic: FP32 deviations from
// the FP64 face average): out[0] += decisions (3 per scalar core, 30 per
// face), out[1] += decisions that differ.
template <int AX>
__device__ __forceinline__ void teno_flips_face(const GridView& g, const double* q, int i, int j, int k,
                                                unsigned long long& dec, unsigned long long& flips) {
    constexpr int NST = 6, CL = 2;
    double st[NST][5];
    const int n = g.n[AX];
    int base_idx[3] = {i, j, k};
    for (int s = 0; s < NST; ++s) {
        int c[3] = {base_idx[0], base_idx[1], base_idx[2]};
        c[AX] = map_index(base_idx[AX] - 3 + s, n, g.bc_lo[AX], g.bc_hi[AX]);
        const long long node = ((long long)c[2] * g.n[1] + c[1]) * g.n[0] + c[0];
        for (int v = 0; v < 5; ++v) st[s][v] = q[v * g.vs + node];
    }
    double qbar[5];
    float qbar32[5];
    for (int v = 0; v < 5; ++v) {
        qbar[v] = 0.5 * (st[CL][v] + st[CL + 1][v]);
        qbar32[v] = float(qbar[v]);
    }
    Eigen<double> e64;
    Eigen<float> e32;
    eigen_at<AX, double>(qbar, g.gamma, e64);
    eigen_at<AX, float>(qbar32, float(g.gamma), e32);
    double c64[NST][5];
    float c32[NST][5];
    for (int s = 0; s < NST; ++s) {
        float d[5];
        for (int v = 0; v < 5; ++v) d[v] = float(st[s][v] - qbar[v]);
        to_characteristic<AX, double>(e64, st[s], c64[s]);
        to_characteristic<AX, float>(e32, d, c32[s]);
    }
    unsigned fl = 0;
    for (int v = 0; v < 5; ++v) {
        // FP32: the (left, right) stencil pair through the paired indicators
        // and cut-off of the FP32-flux kernels
        float2 b2[5], B[3], q[3], keep[3];
        for (int s = 0; s < 5; ++s) b2[s] = make_float2(c32[s][v], c32[NST - 1 - s][v]);
        stencil5x2(b2, B, q);
        float2 bad = make_float2(0.f, 0.f);
        teno_keep32x2(B[0], B[1], B[2], keep, bad);
        flag_bad(bad, fl);
        for (int side = 0; side < 2; ++side) {
            double a[5];
            for (int s = 0; s < 5; ++s) a[s] = side ? c64[NST - 1 - s][v] : c64[s][v];
            double a0, a1, a2;
            teno_betas<double>(a, a0, a1, a2);
            const int m64 = Teno<double>::keep_mask(a0, a1, a2, fl);
            int m32 = 0;
            for (int k = 0; k < 3; ++k) m32 |= int((side ? keep[k].y : keep[k].x) != 0.f) << k;
            dec += 3;
            flips += __popc(m64 ^ m32);
        }
    }
}

__global__ void teno_flips_kernel(GridView g, const double* q, unsigned long long* out) {
    unsigned long long dec = 0, flips = 0;
    const long long cx = g.hi[0] - g.lo[0], cy = g.hi[1] - g.lo[1], cz = g.hi[2] - g.lo[2];
    for (int ax = 0; ax < g.dim; ++ax) {
        // faces between node f-1 and f for f in [lo, hi] along ax, solved nodes across
        const long long fa = (ax == 0 ? cx : (ax == 1 ? cy : cz)) + 1;
        const long long total = fa * (ax == 0 ? cy * cz : (ax == 1 ? cx * cz : cx * cy));
        for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
             t += (long long)gridDim.x * blockDim.x) {
            int i, j, k;
            if (ax == 0) {
                i = g.lo[0] + (int)(t % fa);
                j = g.lo[1] + (int)((t / fa) % cy);
                k = g.lo[2] + (int)(t / (fa * cy));
                teno_flips_face<0>(g, q, i, j, k, dec, flips);
            } else if (ax == 1) {
                i = g.lo[0] + (int)(t % cx);
                j = g.lo[1] + (int)((t / cx) % fa);
                k = g.lo[2] + (int)(t / (cx * fa));
                teno_flips_face<1>(g, q, i, j, k, dec, flips);
            } else {
                i = g.lo[0] + (int)(t % cx);
                j = g.lo[1] + (int)((t / cx) % cy);
                k = g.lo[2] + (int)(t / (cx * cy));
                teno_flips_face<2>(g, q, i, j, k, dec, flips);
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        dec += __shfl_xor_sync(0xffffffffu, dec, o);
        flips += __shfl_xor_sync(0xffffffffu, flips, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(out, dec);
        atomicAdd(out + 1, flips);
    }
}

cudaError_t launch_teno_flips(const GridView& g, const double* q, unsigned long long* out, cudaStream_t st) {
    teno_flips_kernel<<<148 * 4, 256, 0, st>>>(g, q, out);
    return cudaGetLastError();
}

}  // namespace sfg

namespace {

template <typename T>
__global__ void __launch_bounds__(256) fma_chain_kernel(T* out, long long iters, T a, T b) {
    T x0 = T(threadIdx.x) * T(1e-3), x1 = x0 + T(1), x2 = x0 + T(2), x3 = x0 + T(3);
    T x4 = x0 + T(4), x5 = x0 + T(5), x6 = x0 + T(6), x7 = x0 + T(7);
    for (long long i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
            x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
        }
    }
    const T s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (s == T(-1.2345)) out[threadIdx.x] = s;  // keeps the chain alive, never true
}

template <typename T>
int measure(double seconds, double* tflops) {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    T* out = nullptr;
    if (cudaMalloc((void**)&out, 256 * sizeof(T)) != cudaSuccess) return SFG_ERR_NOMEM;
    const int blocks = sms * 8, threads = 256;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    long long iters = 256;
    double best = 0.0;
    for (int round = 0; round < 12; ++round) {
        cudaEventRecord(e0);
        fma_chain_kernel<T><<<blocks, threads>>>(out, iters, T(0.999999), T(1e-7));
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        const double flops = 2.0 * 16 * 8 * (double)iters * blocks * threads;
        const double tf = flops / (ms * 1e-3) / 1e12;
        if (ms > 50.0) best = tf > best ? tf : best;
        if (ms >= seconds * 1e3) break;
        iters = ms > 1.0 ? (long long)(iters * (seconds * 1e3 / ms) * 0.5 + 1) : iters * 8;
        if (iters > (1LL << 34)) iters = 1LL << 34;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return SFG_ERR_CUDA;
    *tflops = best;
    return SFG_OK;
}

}  // namespace

extern "C" int sfg_measure_fma_peak(int fp64, double seconds, double* tflops) {
    if (!tflops) return SFG_ERR_ARG;
    if (!(seconds > 0.0)) seconds = 0.5;
    return fp64 ? measure<double>(seconds, tflops) : measure<float>(seconds, tflops);
}
