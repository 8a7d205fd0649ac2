// sfg_tile.cuh -- fused stage bodies over one tile of nodes, shared by the
// single-grid kernels (sfg_tile2d.cu) and the persistent batched kernels
// (sfg_batch.cu).
//
// A body owns a tile of nodes (TX x TY in 2-D, TX1 in 1-D) whose first node
// is (x0, y0).  It
//   1. stages the tile and its halo (H = NST/2 nodes, cross shape in 2-D)
//      from HBM into shared memory, resolving ghosts by index mapping;
//   2. evaluates every face of the tile once from shared memory into
//      shared-memory flux arrays.  The face list is warp aligned per axis, so
//      no warp mixes the x and y template paths, and sized to whole rounds of
//      256 threads (32 x 15 and 22 x 22 tiles: 4 rounds; 1-D 511 nodes: 2);
//   3. forms div = dFx (+ dFy) per node and finishes it: stage combination
//      with state validation, or R = Jac * div.
// Faces on a tile edge are evaluated by both neighbouring tiles from the same
// inputs, so both see the identical flux and the update stays conservative.
//
// FP32-flux bodies stage the tile as FP32 deviations from the stage's FP64
// reference state (ref_node: the grid's first solved node, the same for every
// tile of a launch): the FP64 -> FP32 rounding happens once per staged node,
// the shared arrays are half the size, and a tile-edge face gets the same
// FP32 inputs, hence the same bits, in both tiles.  Their fluxes are FP32;
// the flux differences (exact: a difference of two floats is exact in
// double), residual and stage update are FP64, so the divergence telescopes
// and the conserved totals drift only at FP64 round-off, as in the FP64 path.
#pragma once

#include <type_traits>

#include "sfg_internal.h"
#include "sfg_math.cuh"
#include "sfg_stage.cuh"

namespace sfg {

constexpr int TILE_THREADS = 256;
constexpr int TILE1D = 511;        // 1-D tile: 512 faces = 2 rounds of 256
constexpr int TILE1D_SHORT = 255;  // 1-D tile of one round (a batch's drained tail)

template <int SCHEME, int TX, int TY>
struct TileShape {
    static constexpr int NST = SchemeInfo<SCHEME>::NST;
    static constexpr int H = NST / 2;
    static constexpr int SX = TX + 2 * H, SY = TY + 2 * H;
    static constexpr int NFX = TY * (TX + 1), NFY = (TY + 1) * TX;
    static constexpr int NFXP = (NFX + 31) / 32 * 32, NFYP = (NFY + 31) / 32 * 32;
    static constexpr int ELEMS = 5 * SX * SY + 5 * NFX + 5 * NFY;  // shared elements
};

template <int SCHEME, int T1 = TILE1D>
struct Tile1Shape {
    static constexpr int NST = SchemeInfo<SCHEME>::NST;
    static constexpr int H = NST / 2;
    static constexpr int SX = T1 + 2 * H;
    static constexpr int NF = T1 + 1;
    static constexpr int ELEMS = 5 * SX + 5 * NF;
};

// Halo index mapping for tile loads.  A partial tile at the high end of an
// axis reaches up to TX - 1 + H nodes past the last node, which can exceed
// one period on small periodic grids, so periodic indices wrap by one period
// and fall back to a full modulo only when that is not enough (both ends are
// periodic or neither; an integer modulo by a run-time n costs tens of
// instructions); transmissive ends clamp to the inner neighbour of the
// boundary node, frozen ends to their extra end node.  Every result lies in
// [0, n).
__device__ __forceinline__ int map_tile_index(int i, int n, int bcl, int bch) {
    if (bcl == BC_PERIODIC) {
        if (i < 0) i += n;
        else if (i >= n) i -= n;
        if ((unsigned)i >= (unsigned)n) {
            i %= n;
            i = i < 0 ? i + n : i;
        }
        return i;
    }
    const int lo = bcl == BC_FROZEN ? 0 : 1;
    const int hi = bch == BC_FROZEN ? n - 1 : n - 2;
    return i < lo ? lo : (i > hi ? hi : i);
}

// Stages the tile and its cross-shaped halo row by row: a warp takes whole
// rows, a lane the columns lane, lane + 32, ...  A lane maps its columns'
// global indices once and a row's index once per row, and the loads of a row
// are coalesced.  put(t, at) stores node `at` of the grid into shared slot t
// (t = r * SX + c).
template <int TX, int TY, int H, typename Put>
__device__ __forceinline__ void stage_rows(const GridView& g, int x0, int y0, Put put) {
    constexpr int SX = TX + 2 * H, SY = TY + 2 * H;
    constexpr int CH = (SX + 31) / 32;  // column chunks of a row
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    int gx[CH];
#pragma unroll
    for (int k = 0; k < CH; ++k)
        gx[k] = map_tile_index(x0 - H + min(lane + 32 * k, SX - 1), g.n[0], g.bc_lo[0], g.bc_hi[0]);
    const long long nx = g.n[0];
    for (int r = warp; r < SY; r += nwarps) {
        const bool band = r >= H && r < TY + H;  // corners are never read
        const long long row = (long long)map_tile_index(y0 - H + r, g.n[1], g.bc_lo[1], g.bc_hi[1]) * nx;
#pragma unroll
        for (int k = 0; k < CH; ++k) {
            const int c = lane + 32 * k;
            if (c >= SX || (!band && (c < H || c >= TX + H))) continue;
            put(r * SX + c, row + gx[k]);
        }
    }
}

// ------------------------------------------------------------------ 2-D FP64
template <int SCHEME, int FLUX, int TX, int TY>
__device__ __forceinline__ void tile2d_body(const GridView& g, const StageView& sv, int x0, int y0, double* smem,
                                            unsigned& flags, unsigned& cut, unsigned& cores, double& sr_max) {
    using S = TileShape<SCHEME, TX, TY>;
    constexpr int NST = S::NST, H = S::H, SX = S::SX, SY = S::SY, NFX = S::NFX, NFY = S::NFY;
    constexpr int NFXP = S::NFXP, NFYP = S::NFYP;
    double* sq = smem;               // [5][SY][SX]
    double* fx = sq + 5 * SX * SY;   // [5][TY][TX+1]
    double* fy = fx + 5 * NFX;       // [5][TY+1][TX]
    const long long nx = g.n[0], vs = g.vs;
    stage_rows<TX, TY, H>(g, x0, y0, [&](int t, long long at) {
        double q[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) q[v] = __ldg(sv.qs + v * vs + at);
#pragma unroll
        for (int v = 0; v < 5; ++v) sq[v * SX * SY + t] = q[v];
    });
    __syncthreads();
    const double gamma = g.gamma;
    for (int f = threadIdx.x; f < NFXP + NFYP; f += blockDim.x) {
        double st[NST][5];
        double Ft[5];
        if (f < NFXP) {
            if (f >= NFX) continue;
            const int r = f / (TX + 1), c = f - r * (TX + 1);
            const double* base = sq + (r + H) * SX + c;  // stencil columns c-H .. c+H-1
#pragma unroll
            for (int s = 0; s < NST; ++s)
#pragma unroll
                for (int v = 0; v < 5; ++v) st[s][v] = base[v * SX * SY + s];
            face_flux<0, SCHEME, FLUX, double>(st, gamma, Ft, flags, cut, FLUX == LAXW ? sv.clock->dt / g.h[0] : 0.0);
#pragma unroll
            for (int v = 0; v < 5; ++v) fx[v * NFX + f] = Ft[v] * g.area[0];
        } else {
            const int k = f - NFXP;
            if (k >= NFY) continue;
            const int r = k / TX, c = k - r * TX;
            const double* base = sq + r * SX + (c + H);  // stencil rows r-H .. r+H-1
#pragma unroll
            for (int s = 0; s < NST; ++s)
#pragma unroll
                for (int v = 0; v < 5; ++v) st[s][v] = base[v * SX * SY + s * SX];
            face_flux<1, SCHEME, FLUX, double>(st, gamma, Ft, flags, cut, FLUX == LAXW ? sv.clock->dt / g.h[1] : 0.0);
#pragma unroll
            for (int v = 0; v < 5; ++v) fy[v * NFY + k] = Ft[v] * g.area[1];
        }
        if (SCHEME == TENO5) cores += 10;
    }
    __syncthreads();
    const double dt = sv.clock->dt;
    for (int n = threadIdx.x; n < TX * TY; n += blockDim.x) {
        const int r = n / TX, c = n - r * TX;
        const int gx = x0 + c, gy = y0 + r;
        if (gx >= g.hi[0] || gy >= g.hi[1]) continue;
        const long long node = (long long)gy * nx + gx;
        double div[5], qn[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            const double* fxv = fx + v * NFX + r * (TX + 1) + c;
            const double* fyv = fy + v * NFY + r * TX + c;
            div[v] = (fxv[1] - fxv[0]) + (fyv[TX] - fyv[0]);
            qn[v] = sq[v * SX * SY + (r + H) * SX + c + H];
        }
        finish_node(g, sv, dt, node, qn, div, flags, sr_max);
    }
}

// ------------------------------------------------------------------ 2-D FP32 flux
template <int SCHEME, int FLUX, int TX, int TY>
__device__ __forceinline__ void tile2d_f32_body(const GridView& g, const StageView& sv, int x0, int y0, float* smem,
                                                unsigned& flags, unsigned& cut, unsigned& cores, double& sr_max) {
    using S = TileShape<SCHEME, TX, TY>;
    constexpr int NST = S::NST, H = S::H, SX = S::SX, SY = S::SY, NFX = S::NFX, NFY = S::NFY;
    constexpr int NFXP = S::NFXP, NFYP = S::NFYP;
    float* sq = smem;               // [5][SY][SX] deviations from qref
    float* fx = sq + 5 * SX * SY;   // [5][TY][TX+1]
    float* fy = fx + 5 * NFX;       // [5][TY+1][TX]
    const long long nx = g.n[0], vs = g.vs;
    // the FP32 reference (velocity, pressure) is made once per tile by one
    // thread; every face reads it after the staging barrier (the previous
    // tile's faces are all done before thread 0 gets here again)
    __shared__ Ref32 sref;
    double qref[5];
    load_ref(g, sv.qs, qref);
    if (threadIdx.x == 0) sref = make_ref32(qref, g.gamma);
    stage_rows<TX, TY, H>(g, x0, y0, [&](int t, long long at) {
        double q[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) q[v] = __ldg(sv.qs + v * vs + at);
#pragma unroll
        for (int v = 0; v < 5; ++v) sq[v * SX * SY + t] = float(q[v] - qref[v]);
    });
    __syncthreads();
    const Ref32 ref = sref;
    const float gamma = float(g.gamma);
    for (int f = threadIdx.x; f < NFXP + NFYP; f += blockDim.x) {
        float st[NST][5];
        float Ft[5];
        if (f < NFXP) {
            if (f >= NFX) continue;
            const int r = f / (TX + 1), c = f - r * (TX + 1);
            const float* base = sq + (r + H) * SX + c;
#pragma unroll
            for (int s = 0; s < NST; ++s)
#pragma unroll
                for (int v = 0; v < 5; ++v) st[s][v] = base[v * SX * SY + s];
            face_flux_dev32<0, SCHEME, FLUX>(st, ref, gamma, Ft, flags, cut, sv.counters != nullptr,
                                             float(g.area[0]));
#pragma unroll
            for (int v = 0; v < 5; ++v) fx[v * NFX + f] = Ft[v];
        } else {
            const int k = f - NFXP;
            if (k >= NFY) continue;
            const int r = k / TX, c = k - r * TX;
            const float* base = sq + r * SX + (c + H);
#pragma unroll
            for (int s = 0; s < NST; ++s)
#pragma unroll
                for (int v = 0; v < 5; ++v) st[s][v] = base[v * SX * SY + s * SX];
            face_flux_dev32<1, SCHEME, FLUX>(st, ref, gamma, Ft, flags, cut, sv.counters != nullptr,
                                             float(g.area[1]));
#pragma unroll
            for (int v = 0; v < 5; ++v) fy[v * NFY + k] = Ft[v];
        }
        if (SCHEME == TENO5) cores += 10;
    }
    __syncthreads();
    const double dt = sv.clock->dt;
    for (int n = threadIdx.x; n < TX * TY; n += blockDim.x) {
        const int r = n / TX, c = n - r * TX;
        const int gx = x0 + c, gy = y0 + r;
        if (gx >= g.hi[0] || gy >= g.hi[1]) continue;
        const long long node = (long long)gy * nx + gx;
        double div[5], qn[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            const float* fxv = fx + v * NFX + r * (TX + 1) + c;
            const float* fyv = fy + v * NFY + r * TX + c;
            // FP32 face values, differences in FP64: the difference of two
            // floats is exact in double, so the divergence telescopes
            div[v] = (double(fxv[1]) - double(fxv[0])) + (double(fyv[TX]) - double(fyv[0]));
            qn[v] = __ldg(sv.qs + v * vs + node);
        }
        finish_node(g, sv, dt, node, qn, div, flags, sr_max);
    }
}

// ------------------------------------------------------------------ 1-D
// T = double: FP64 stencil; T = float: FP32 deviations from the stage's reference node.
// T1 nodes per tile; every face and node gets the same bits whatever the
// tile length (the FP32 reference is the stage's, not the tile's).
template <int SCHEME, int FLUX, typename T, int T1 = TILE1D>
__device__ __forceinline__ void tile1d_body(const GridView& g, const StageView& sv, int x0, T* smem, unsigned& flags,
                                            unsigned& cut, unsigned& cores, double& sr_max) {
    using S = Tile1Shape<SCHEME, T1>;
    constexpr int NST = S::NST, H = S::H, SX = S::SX, NF = S::NF;
    constexpr bool F32 = sizeof(T) == sizeof(float);
    T* sq = smem;          // [5][SX]
    T* fx = sq + 5 * SX;   // [5][NF]
    const long long vs = g.vs;
    double qref[5] = {0, 0, 0, 0, 0};
    __shared__ Ref32 sref;  // FP32: made once per tile, read after the staging barrier
    if (F32) {
        load_ref(g, sv.qs, qref);
        if (threadIdx.x == 0) sref = make_ref32(qref, g.gamma);
    }
    for (int t = threadIdx.x; t < SX; t += blockDim.x) {
        const int gx = map_tile_index(x0 - H + t, g.n[0], g.bc_lo[0], g.bc_hi[0]);
#pragma unroll
        for (int v = 0; v < 5; ++v) sq[v * SX + t] = T(__ldg(sv.qs + v * vs + gx) - qref[v]);
    }
    __syncthreads();
    const Ref32 ref = F32 ? sref : Ref32{};
    for (int f = threadIdx.x; f < NF; f += blockDim.x) {
        T st[NST][5];
        T Ft[5];
#pragma unroll
        for (int s = 0; s < NST; ++s)
#pragma unroll
            for (int v = 0; v < 5; ++v) st[s][v] = sq[v * SX + f + s];
        if constexpr (F32) {
            face_flux_dev32<0, SCHEME, FLUX>(st, ref, T(g.gamma), Ft, flags, cut, sv.counters != nullptr,
                                             T(g.area[0]));
#pragma unroll
            for (int v = 0; v < 5; ++v) fx[v * NF + f] = Ft[v];
        } else {
            face_flux<0, SCHEME, FLUX, double>(st, g.gamma, Ft, flags, cut, FLUX == LAXW ? sv.clock->dt / g.h[0] : 0.0);
#pragma unroll
            for (int v = 0; v < 5; ++v) fx[v * NF + f] = Ft[v] * T(g.area[0]);
        }
        if (SCHEME == TENO5) cores += 10;
    }
    __syncthreads();
    const double dt = sv.clock->dt;
    for (int c = threadIdx.x; c < T1; c += blockDim.x) {
        const int gx = x0 + c;
        if (gx >= g.hi[0]) continue;
        double div[5], qn[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            div[v] = double(fx[v * NF + c + 1]) - double(fx[v * NF + c]);  // FP32 faces: exact FP64 difference
            qn[v] = F32 ? __ldg(sv.qs + v * vs + gx) : double(sq[v * SX + c + H]);
        }
        finish_node(g, sv, dt, gx, qn, div, flags, sr_max);
    }
}

}  // namespace sfg
