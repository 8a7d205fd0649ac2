// sfg_laws.cu -- physical boundary laws of SFG_BC_LAW ends: fixedValue,
// zeroGradient and symmetry for density, velocity and pressure, with the
// energy rebuilt from pressure (Boundary::Applicator::apply,
// solver/boundary/SF_applicator.h:51-83).
//
// One thread per boundary point of a law end whose other coordinates lie in
// the solved range.  Every ghost layer of the reference derives from the
// boundary node alone (forBoundaryGhostsAlongAxis, SF_boundary.h:95-121), so
// all layers hold one value: the end's extra node.  Points on two law faces
// (box edges and corners) are read by no stencil of a solved node and are
// left as they are.
//
// The reference reads densities and pressures of some points through the
// Field's thermodynamic state cache (Field::thermodynamicState,
// SF_field.cpp:133-151), which its own writes do not refresh: the velocity
// fixedValue law caches the boundary node's state after the density write and
// before the momentum and energy writes, and the pressure law then reads that
// state's pressure for the ghosts.  The table has min(storage points, 4096)
// direct-mapped entries, so on larger Fields another point's query can evict
// that entry first: the pressure law then closes the boundary node afresh,
// or (evicted inside the velocity law's own ghost loop) sees the new momentum
// with the old energy.  Which of the three a point reads depends only on the
// grid and the laws; the host replays the reference's query sequence once
// (simulate_law_cache) and hands the kernel one code per point (lv.codes).
// The kernel builds that state from the boundary node's value before this
// application (`old`).
//
// Arithmetic is FP64 with explicit round-to-nearest intrinsics in the
// reference's operation order (no contraction), so the values equal the
// oracle's bit for bit.
#include "sfg_laws.cuh"

namespace sfg {

__global__ void __launch_bounds__(128) law_fill_kernel(GridView g, LawView lv, const double* old, double* q,
                                                         const Clock* clock,
                                                         int require_active, unsigned* flags) {
    if (require_active && !clock->active) return;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= lv.start[lv.count]) return;
    law_fill_point(g, lv, old, q, t, flags);
}

cudaError_t launch_law_fill(const GridView& g, const LawView& lv, const double* old, double* q, const Clock* clock,
                            int require_active, unsigned* flags, cudaStream_t st) {
    const long long points = lv.start[lv.count];
    if (points <= 0) return cudaSuccess;
    law_fill_kernel<<<(unsigned)((points + 127) / 128), 128, 0, st>>>(g, lv, old, q, clock, require_active, flags);
    return cudaGetLastError();
}

}  // namespace sfg
