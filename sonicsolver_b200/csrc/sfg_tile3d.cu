// sfg_tile3d.cu -- fused stage kernel for 3-D grids: one launch per stage.
//
// A block owns a column of nodes TX x TY (x, y) by up to KZ planes (z) and
// marches up the planes.  Per plane k it
//   1. stages plane k+H of its TX x TY interior into a ring of 2H planes
//      (the z stencils of the block's columns), and plane k with its x-y halo
//      (cross shape, H deep) into a plane buffer;
//   2. evaluates the x and y faces of plane k from the plane buffer into
//      shared flux arrays (TY (TX + 1) + (TY + 1) TX = 511 faces for
//      16 x 15: two rounds of 256 threads), and, one per thread and column,
//      the z face k + 1/2 from the ring; the face k - 1/2 carries over from
//      the previous plane in registers;
//   3. finishes the plane's nodes (stage update, or R = Jac div).
// Ghosts and periodic images come from index mapping, as in the 2-D tiles.
// A face on a block edge (x, y, or the bottom z face of a chunk) is
// evaluated by both neighbouring blocks from the same inputs.
//
// T = double: FP64 stencils.  T = float: FP32 deviations from the stage's
// reference node (ref_node; one FP64 -> FP32 rounding per staged node) and
// deviation fluxes (face_flux_dev32): the reference flux cancels from every
// flux difference, and a block-edge face has the same bits in both blocks.
// Divergence (exact FP64 differences of the FP32 faces) and stage update
// are FP64.
#include "sfg_tile.cuh"

namespace sfg {

constexpr int T3X = 16, T3Y = 15, T3Z = 32;
// resident CTAs per SM of the FP32 kernel: 64 registers a thread and 48 KB
// of shared memory each (with the full shared-memory carveout)
constexpr int T3_F32_CTAS = 4;

template <int SCHEME, typename T>
struct Tile3Shape {
    static constexpr int NST = SchemeInfo<SCHEME>::NST;
    static constexpr int H = NST / 2;
    static constexpr int R = 2 * H;                        // ring planes
    static constexpr int COL = T3X * T3Y;                  // columns (240)
    static constexpr int SX = T3X + 2 * H, SY = T3Y + 2 * H;
    static constexpr int NFX = T3Y * (T3X + 1), NFY = (T3Y + 1) * T3X;
    static constexpr int ELEMS = 5 * R * COL + 5 * SX * SY + 5 * NFX + 5 * NFY;
};

template <int SCHEME, int FLUX, typename T>
__global__ void __launch_bounds__(TILE_THREADS, sizeof(T) == sizeof(float) ? T3_F32_CTAS : 2)
    tile3d_kernel(GridView g, StageView sv) {
    using S = Tile3Shape<SCHEME, T>;
    constexpr int NST = S::NST, H = S::H, R = S::R, COL = S::COL, SX = S::SX, SY = S::SY;
    constexpr int NFX = S::NFX, NFY = S::NFY;
    constexpr bool F32 = sizeof(T) == sizeof(float);
    extern __shared__ __align__(16) unsigned char smem3[];
    T* ring = reinterpret_cast<T*>(smem3);  // [5][R][COL]
    T* box = ring + 5 * R * COL;            // [5][SY][SX] plane k with its x-y halo
    T* fx = box + 5 * SX * SY;              // [5][TY][TX+1]
    T* fy = fx + 5 * NFX;                   // [5][TY+1][TX]
    if (sv.require_active && !sv.clock->active) return;

    const int ntx = (g.hi[0] - g.lo[0] + T3X - 1) / T3X;
    const int nty = (g.hi[1] - g.lo[1] + T3Y - 1) / T3Y;
    const int bxy = blockIdx.x % (ntx * nty), bz = blockIdx.x / (ntx * nty);
    const int x0 = g.lo[0] + (bxy % ntx) * T3X, y0 = g.lo[1] + (bxy / ntx) * T3Y;
    const int z0 = g.lo[2] + bz * T3Z, z1 = min(z0 + T3Z, g.hi[2]);
    const long long nx = g.n[0], nxy = (long long)g.n[0] * g.n[1], vs = g.vs;
    const int t = threadIdx.x;
    const int ci = t % T3X, cj = t / T3X;  // this thread's column (t < COL)

    // reference state of the stage (FP32 deviations), none in FP64
    double qref[5] = {0, 0, 0, 0, 0};
    if (F32) load_ref(g, sv.qs, qref);
    const Ref32 ref = F32 ? make_ref32(qref, g.gamma) : Ref32{};
    auto load = [&](long long at, int v) -> T { return T(__ldg(sv.qs + v * vs + at) - qref[v]); };

    // stage plane p of the block's interior into its ring slot
    auto stage_ring = [&](int p) {
        const int zk = map_tile_index(p, g.n[2], g.bc_lo[2], g.bc_hi[2]);
        const int slot = ((p % R) + R) % R;
        for (int c = t; c < COL; c += blockDim.x) {
            const int gx = map_tile_index(x0 + c % T3X, g.n[0], g.bc_lo[0], g.bc_hi[0]);
            const int gy = map_tile_index(y0 + c / T3X, g.n[1], g.bc_lo[1], g.bc_hi[1]);
            const long long at = (long long)zk * nxy + (long long)gy * nx + gx;
#pragma unroll
            for (int v = 0; v < 5; ++v) ring[(v * R + slot) * COL + c] = load(at, v);
        }
    };
    // z face p + 1/2 of this thread's column from ring planes p+1-H .. p+H
    auto z_face = [&](int p, T Fz[5], unsigned& flags, unsigned& cut) {
        if constexpr (F32) {
            float d[NST][5];
#pragma unroll
            for (int s = 0; s < NST; ++s) {
                const int slot = (((p + 1 - H + s) % R) + R) % R;
#pragma unroll
                for (int v = 0; v < 5; ++v) d[s][v] = ring[(v * R + slot) * COL + t];
            }
            face_flux_dev32<2, SCHEME, FLUX>(d, ref, float(g.gamma), Fz, flags, cut, sv.counters != nullptr);
        } else {
            double st[NST][5];
#pragma unroll
            for (int s = 0; s < NST; ++s) {
                const int slot = (((p + 1 - H + s) % R) + R) % R;
#pragma unroll
                for (int v = 0; v < 5; ++v) st[s][v] = ring[(v * R + slot) * COL + t];
            }
            face_flux<2, SCHEME, FLUX, double>(st, g.gamma, Fz, flags, cut,
                                               FLUX == LAXW ? sv.clock->dt / g.h[2] : 0.0);
        }
    };

    unsigned flags = 0, cut = 0, cores = 0;
    double sr = 0.0;
    // prologue: ring planes z0-H .. z0+H-1, then the face z0 - 1/2
    for (int p = z0 - H; p < z0 + H; ++p) stage_ring(p);
    __syncthreads();
    T Fdn[5] = {0, 0, 0, 0, 0};
    if (t < COL) z_face(z0 - 1, Fdn, flags, cut);
    const double dt = sv.clock->dt;
    const T lamx = T(FLUX == LAXW ? sv.clock->dt / g.h[0] : 0.0);
    const T lamy = T(FLUX == LAXW ? sv.clock->dt / g.h[1] : 0.0);

    for (int k = z0; k < z1; ++k) {
        __syncthreads();  // previous plane's faces and z stencils are consumed
        stage_ring(k + H);
        // plane k with its x-y halo (interior from the ring)
        const int zk = map_tile_index(k, g.n[2], g.bc_lo[2], g.bc_hi[2]);
        const int slot_k = ((k % R) + R) % R;
        for (int e = t; e < SX * SY; e += blockDim.x) {
            const int r = e / SX, c = e - r * SX;
            const bool in_x = c >= H && c < T3X + H, in_y = r >= H && r < T3Y + H;
            if (!in_x && !in_y) continue;  // corners are never read
            if (in_x && in_y) {
                const int col = (r - H) * T3X + (c - H);
#pragma unroll
                for (int v = 0; v < 5; ++v) box[v * SX * SY + e] = ring[(v * R + slot_k) * COL + col];
            } else {
                const int gx = map_tile_index(x0 - H + c, g.n[0], g.bc_lo[0], g.bc_hi[0]);
                const int gy = map_tile_index(y0 - H + r, g.n[1], g.bc_lo[1], g.bc_hi[1]);
                const long long at = (long long)zk * nxy + (long long)gy * nx + gx;
#pragma unroll
                for (int v = 0; v < 5; ++v) box[v * SX * SY + e] = load(at, v);
            }
        }
        __syncthreads();
        // x and y faces of plane k (faces f < NFX are x faces)
        for (int f = t; f < NFX + NFY; f += blockDim.x) {
            T st[NST][5];
            T Ft[5];
            if (f < NFX) {
                const int r = f / (T3X + 1), c = f - r * (T3X + 1);
                const T* base = box + (r + H) * SX + c;
#pragma unroll
                for (int s = 0; s < NST; ++s)
#pragma unroll
                    for (int v = 0; v < 5; ++v) st[s][v] = base[v * SX * SY + s];
                if constexpr (F32) {
                    // the area rides in the flux's exact factor 1/2
                    face_flux_dev32<0, SCHEME, FLUX>(st, ref, float(g.gamma), Ft, flags, cut, sv.counters != nullptr,
                                                     float(g.area[0]));
#pragma unroll
                    for (int v = 0; v < 5; ++v) fx[v * NFX + f] = Ft[v];
                } else {
                    double sd[NST][5];
#pragma unroll
                    for (int s = 0; s < NST; ++s)
#pragma unroll
                        for (int v = 0; v < 5; ++v) sd[s][v] = st[s][v];
                    face_flux<0, SCHEME, FLUX, double>(sd, g.gamma, Ft, flags, cut, lamx);
#pragma unroll
                    for (int v = 0; v < 5; ++v) fx[v * NFX + f] = Ft[v] * T(g.area[0]);
                }
            } else {
                const int kf = f - NFX;
                const int r = kf / T3X, c = kf - r * T3X;
                const T* base = box + r * SX + (c + H);
#pragma unroll
                for (int s = 0; s < NST; ++s)
#pragma unroll
                    for (int v = 0; v < 5; ++v) st[s][v] = base[v * SX * SY + s * SX];
                if constexpr (F32) {
                    // the area rides in the flux's exact factor 1/2
                    face_flux_dev32<1, SCHEME, FLUX>(st, ref, float(g.gamma), Ft, flags, cut, sv.counters != nullptr,
                                                     float(g.area[1]));
#pragma unroll
                    for (int v = 0; v < 5; ++v) fy[v * NFY + kf] = Ft[v];
                } else {
                    double sd[NST][5];
#pragma unroll
                    for (int s = 0; s < NST; ++s)
#pragma unroll
                        for (int v = 0; v < 5; ++v) sd[s][v] = st[s][v];
                    face_flux<1, SCHEME, FLUX, double>(sd, g.gamma, Ft, flags, cut, lamy);
#pragma unroll
                    for (int v = 0; v < 5; ++v) fy[v * NFY + kf] = Ft[v] * T(g.area[1]);
                }
            }
            if (SCHEME == TENO5) cores += 10;
        }
        T Fup[5] = {0, 0, 0, 0, 0};
        if (t < COL) {
            z_face(k, Fup, flags, cut);
            if (SCHEME == TENO5) cores += 10;
        }
        __syncthreads();
        // finish plane k
        if (t < COL && x0 + ci < g.hi[0] && y0 + cj < g.hi[1]) {
            const long long node = (long long)k * nxy + (long long)(y0 + cj) * nx + (x0 + ci);
            double div[5], qn[5];
#pragma unroll
            for (int v = 0; v < 5; ++v) {
                const T* fxv = fx + v * NFX + cj * (T3X + 1) + ci;
                const T* fyv = fy + v * NFY + cj * T3X + ci;
                if constexpr (F32)  // FP32 face values, exact FP64 differences
                    div[v] = (double(fxv[1]) - double(fxv[0])) + (double(fyv[T3X]) - double(fyv[0])) +
                             (double(Fup[v]) - double(Fdn[v])) * g.area[2];
                else
                    div[v] = (fxv[1] - fxv[0]) + (fyv[T3X] - fyv[0]) + (Fup[v] * g.area[2] - Fdn[v] * g.area[2]);
                qn[v] = __ldg(sv.qs + v * vs + node);
            }
            finish_node(g, sv, dt, node, qn, div, flags, sr);
        }
#pragma unroll
        for (int v = 0; v < 5; ++v) Fdn[v] = Fup[v];
    }
    flush_status(sv, flags, cores, cut);
    if (sv.mode & MODE_CFL) flush_cfl_block(g, sv.clock, sr);
}

template <int SCHEME, int FLUX, typename T>
static cudaError_t launch_tile3(const GridView& g, const StageView& sv, cudaStream_t st) {
    constexpr size_t smem = sizeof(T) * Tile3Shape<SCHEME, T>::ELEMS;
    static std::atomic<unsigned long long> configured{0};
    unsigned long long bit = 0;
    auto kern = tile3d_kernel<SCHEME, FLUX, T>;
    if (attributes_pending(configured, bit)) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        // the whole unified L1 / shared array as shared memory: four FP32
        // CTAs of 48 KB per SM
        e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
        if (e != cudaSuccess) return e;
        configured.fetch_or(bit, std::memory_order_release);
    }
    const int ntx = (g.hi[0] - g.lo[0] + T3X - 1) / T3X;
    const int nty = (g.hi[1] - g.lo[1] + T3Y - 1) / T3Y;
    const int ntz = (g.hi[2] - g.lo[2] + T3Z - 1) / T3Z;
    kern<<<ntx * nty * ntz, TILE_THREADS, smem, st>>>(g, sv);
    return cudaGetLastError();
}

template <int FLUX, typename T>
static cudaError_t launch_tile3_s(int scheme, const GridView& g, const StageView& sv, cudaStream_t st) {
    switch (scheme) {
    case WENO5: return launch_tile3<WENO5, FLUX, T>(g, sv, st);
    case TENO5: return launch_tile3<TENO5, FLUX, T>(g, sv, st);
    case WENO3: return launch_tile3<WENO3, FLUX, T>(g, sv, st);
    case WENO7: return launch_tile3<WENO7, FLUX, T>(g, sv, st);
    }
    return cudaErrorInvalidValue;
}

template <typename T>
static cudaError_t launch_tile3_t(int scheme, int flux, const GridView& g, const StageView& sv, cudaStream_t st) {
    if (flux == RUSANOV) return launch_tile3_s<RUSANOV, T>(scheme, g, sv, st);
    if (flux == ROE) return launch_tile3_s<ROE, T>(scheme, g, sv, st);
    if constexpr (sizeof(T) == sizeof(double)) {
        if (flux == STEGER) return launch_tile3_s<STEGER, T>(scheme, g, sv, st);
        if (flux == LAXF) return launch_tile3_s<LAXF, T>(scheme, g, sv, st);
        if (flux == LAXW) return launch_tile3_s<LAXW, T>(scheme, g, sv, st);
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_tile3d(int scheme, int flux, int prec64, const GridView& g, const StageView& sv, cudaStream_t st) {
    return prec64 ? launch_tile3_t<double>(scheme, flux, g, sv, st) : launch_tile3_t<float>(scheme, flux, g, sv, st);
}

}  // namespace sfg
