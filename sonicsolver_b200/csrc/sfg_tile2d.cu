// sfg_tile2d.cu -- single-grid fused stage kernels for 2-D grids: one launch
// per stage, one block per tile (bodies in sfg_tile.cuh).
#include "sfg_tile.cuh"

namespace sfg {

template <int SCHEME, int FLUX, int TX, int TY>
__global__ void __launch_bounds__(TILE_THREADS, 2) tile2d_kernel(GridView g, StageView sv) {
    extern __shared__ __align__(16) double smem[];
    if (sv.require_active && !sv.clock->active) return;
    const int ntx = (g.hi[0] - g.lo[0] + TX - 1) / TX;
    const int x0 = g.lo[0] + (blockIdx.x % ntx) * TX, y0 = g.lo[1] + (blockIdx.x / ntx) * TY;
    unsigned flags = 0, cut = 0, cores = 0;
    double sr = 0.0;
    tile2d_body<SCHEME, FLUX, TX, TY>(g, sv, x0, y0, smem, flags, cut, cores, sr);
    flush_status(sv, flags, cores, cut);
    if (sv.mode & MODE_CFL) flush_cfl_block(g, sv.clock, sr);
}

template <int SCHEME, int FLUX, int TX, int TY>
__global__ void __launch_bounds__(TILE_THREADS, 4) tile2d_f32_kernel(GridView g, StageView sv) {
    extern __shared__ __align__(16) float smemf[];
    if (sv.require_active && !sv.clock->active) return;
    const int ntx = (g.hi[0] - g.lo[0] + TX - 1) / TX;
    const int x0 = g.lo[0] + (blockIdx.x % ntx) * TX, y0 = g.lo[1] + (blockIdx.x / ntx) * TY;
    unsigned flags = 0, cut = 0, cores = 0;
    double sr = 0.0;
    tile2d_f32_body<SCHEME, FLUX, TX, TY>(g, sv, x0, y0, smemf, flags, cut, cores, sr);
    flush_status(sv, flags, cores, cut);
    if (sv.mode & MODE_CFL) flush_cfl_block(g, sv.clock, sr);
}

template <int SCHEME, int FLUX, typename T, int TX, int TY>
static cudaError_t launch_tile(const GridView& g, const StageView& sv, cudaStream_t st) {
    using S = TileShape<SCHEME, TX, TY>;
    constexpr size_t smem = sizeof(T) * S::ELEMS;
    static std::atomic<unsigned long long> configured{0};
    unsigned long long bit = 0;
    const int ntx = (g.hi[0] - g.lo[0] + TX - 1) / TX;
    const int nty = (g.hi[1] - g.lo[1] + TY - 1) / TY;
    auto kern = sizeof(T) == sizeof(float) ? tile2d_f32_kernel<SCHEME, FLUX, TX, TY> : tile2d_kernel<SCHEME, FLUX, TX, TY>;
    if (attributes_pending(configured, bit)) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        configured.fetch_or(bit, std::memory_order_release);
    }
    kern<<<ntx * nty, TILE_THREADS, smem, st>>>(g, sv);
    return cudaGetLastError();
}

template <int FLUX, typename T, int TX, int TY>
static cudaError_t launch_tile_s(int scheme, const GridView& g, const StageView& sv, cudaStream_t st) {
    switch (scheme) {
    case WENO5: return launch_tile<WENO5, FLUX, T, TX, TY>(g, sv, st);
    case TENO5: return launch_tile<TENO5, FLUX, T, TX, TY>(g, sv, st);
    case WENO3: return launch_tile<WENO3, FLUX, T, TX, TY>(g, sv, st);
    case WENO7: return launch_tile<WENO7, FLUX, T, TX, TY>(g, sv, st);
    }
    return cudaErrorInvalidValue;
}

// Rusanov and Roe in both precisions; Steger-Warming, Lax-Friedrichs and
// Lax-Wendroff faces in FP64 (the FP32 deviation form is Rusanov / Roe).
template <typename T, int TX, int TY>
static cudaError_t launch_tile_t(int scheme, int flux, const GridView& g, const StageView& sv, cudaStream_t st) {
    if (flux == RUSANOV) return launch_tile_s<RUSANOV, T, TX, TY>(scheme, g, sv, st);
    if (flux == ROE) return launch_tile_s<ROE, T, TX, TY>(scheme, g, sv, st);
    if constexpr (sizeof(T) == sizeof(double)) {
        if (flux == STEGER) return launch_tile_s<STEGER, T, TX, TY>(scheme, g, sv, st);
        if (flux == LAXF) return launch_tile_s<LAXF, T, TX, TY>(scheme, g, sv, st);
        if (flux == LAXW) return launch_tile_s<LAXW, T, TX, TY>(scheme, g, sv, st);
    }
    return cudaErrorInvalidValue;
}

// 1-D grids: one block per 511-node tile (the body the batched kernels use,
// so a 1-D grid gives the same bits alone and in a batch).
template <int SCHEME, int FLUX, typename T>
__global__ void __launch_bounds__(TILE_THREADS) tile1d_kernel(GridView g, StageView sv) {
    extern __shared__ __align__(16) unsigned char smem1[];
    if (sv.require_active && !sv.clock->active) return;
    unsigned flags = 0, cut = 0, cores = 0;
    double sr = 0.0;
    tile1d_body<SCHEME, FLUX, T>(g, sv, g.lo[0] + blockIdx.x * TILE1D, reinterpret_cast<T*>(smem1), flags, cut,
                                 cores, sr);
    flush_status(sv, flags, cores, cut);
    if (sv.mode & MODE_CFL) flush_cfl_block(g, sv.clock, sr);
}

template <int SCHEME, int FLUX, typename T>
static cudaError_t launch_tile1(const GridView& g, const StageView& sv, cudaStream_t st) {
    constexpr size_t smem = sizeof(T) * Tile1Shape<SCHEME>::ELEMS;
    static std::atomic<unsigned long long> configured{0};
    unsigned long long bit = 0;
    auto kern = tile1d_kernel<SCHEME, FLUX, T>;
    if (attributes_pending(configured, bit)) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        configured.fetch_or(bit, std::memory_order_release);
    }
    kern<<<(g.hi[0] - g.lo[0] + TILE1D - 1) / TILE1D, TILE_THREADS, smem, st>>>(g, sv);
    return cudaGetLastError();
}

template <int FLUX, typename T>
static cudaError_t launch_tile1_s(int scheme, const GridView& g, const StageView& sv, cudaStream_t st) {
    switch (scheme) {
    case WENO5: return launch_tile1<WENO5, FLUX, T>(g, sv, st);
    case TENO5: return launch_tile1<TENO5, FLUX, T>(g, sv, st);
    case WENO3: return launch_tile1<WENO3, FLUX, T>(g, sv, st);
    case WENO7: return launch_tile1<WENO7, FLUX, T>(g, sv, st);
    }
    return cudaErrorInvalidValue;
}

template <typename T>
static cudaError_t launch_tile1_t(int scheme, int flux, const GridView& g, const StageView& sv, cudaStream_t st) {
    if (flux == RUSANOV) return launch_tile1_s<RUSANOV, T>(scheme, g, sv, st);
    if (flux == ROE) return launch_tile1_s<ROE, T>(scheme, g, sv, st);
    if constexpr (sizeof(T) == sizeof(double)) {
        if (flux == STEGER) return launch_tile1_s<STEGER, T>(scheme, g, sv, st);
        if (flux == LAXF) return launch_tile1_s<LAXF, T>(scheme, g, sv, st);
        if (flux == LAXW) return launch_tile1_s<LAXW, T>(scheme, g, sv, st);
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_tile1d(int scheme, int flux, int prec64, const GridView& g, const StageView& sv, cudaStream_t st) {
    return prec64 ? launch_tile1_t<double>(scheme, flux, g, sv, st) : launch_tile1_t<float>(scheme, flux, g, sv, st);
}

// variant 1: 32 x 15 tile, variant 2: 22 x 22 tile (256 threads each).
cudaError_t launch_tile2d(int variant, int scheme, int flux, int prec64, const GridView& g, const StageView& sv,
                          cudaStream_t st) {
    if (variant == 1)
        return prec64 ? launch_tile_t<double, 32, 15>(scheme, flux, g, sv, st)
                      : launch_tile_t<float, 32, 15>(scheme, flux, g, sv, st);
    if (variant == 2)
        return prec64 ? launch_tile_t<double, 22, 22>(scheme, flux, g, sv, st)
                      : launch_tile_t<float, 22, 22>(scheme, flux, g, sv, st);
    return cudaErrorInvalidValue;
}

}  // namespace sfg
