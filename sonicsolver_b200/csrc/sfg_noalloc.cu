// sfg_noalloc.cu -- spatial residual of a caller-owned device state, with
// no device allocation (sfg_residual_noalloc in include/sonicsolver_b200.h).
//
// The working memory (the residual accumulated across axis sweeps, the step
// clock the sweeps read and the status word) lives in one file-scope
// __device__ array.  In host code `g_noalloc_scratch` only names a host-side
// shadow of that array, never device memory: a kernel given it would fault or
// silently use the wrong memory.  The device address is looked up once per
// device with cudaGetSymbolAddress and that pointer is what the kernels get.
// The cached address belongs to the device's current context: after
// cudaDeviceReset the module is loaded again and the address may change, so
// the entry point is not valid across a reset in the same process.
#include "../../include/sonicsolver_b200.h"
#include "sfg_internal.h"

#include <cmath>
#include <cstdio>
#include <mutex>
#include <string>

namespace sfg {
cudaError_t launch_sweep(int scheme, int flux, int prec64, int axis, const GridView& g, const StageView& sv,
                         cudaStream_t st);
void set_last_error(const char* msg);
}  // namespace sfg
using namespace sfg;

namespace {

constexpr long long kHeaderDoubles = 32;  // 256 bytes: Clock + status word
static_assert(sizeof(Clock) <= 16 * sizeof(double), "clock must fit the header");

static __device__ __align__(256) double g_noalloc_scratch[kHeaderDoubles + 5LL * SFG_NOALLOC_MAX_NODES];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
double* g_device_address[kMaxDevices] = {};

int noalloc_fail(int code, const char* msg) {
    set_last_error(msg);
    return code;
}

// Device address of the scratch array on the current device (looked up on
// the first call per device).
int scratch_address(double** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return noalloc_fail(SFG_ERR_CUDA, "no current CUDA device");
    if (dev < 0 || dev >= kMaxDevices) return noalloc_fail(SFG_ERR_ARG, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_device_address[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) return noalloc_fail(SFG_ERR_CUDA, cudaGetErrorString(e));
        g_device_address[dev] = static_cast<double*>(p);
    }
    *out = g_device_address[dev];
    return SFG_OK;
}

struct RecipeParts {
    int id, scheme, flux;
};
const RecipeParts kParts[] = {{SFG_RECIPE_WENO3_RUSANOV, WENO3, RUSANOV}, {SFG_RECIPE_WENO3_ROE, WENO3, ROE},
                              {SFG_RECIPE_WENO5_RUSANOV, WENO5, RUSANOV}, {SFG_RECIPE_WENO5_ROE, WENO5, ROE},
                              {SFG_RECIPE_TENO5_RUSANOV, TENO5, RUSANOV}, {SFG_RECIPE_TENO5_ROE, TENO5, ROE},
                              {SFG_RECIPE_WENO7_RUSANOV, WENO7, RUSANOV}, {SFG_RECIPE_WENO7_ROE, WENO7, ROE}};

}  // namespace

extern "C" int sfg_residual_noalloc(const sfg_grid_desc* grid, const sfg_numerics_desc* numerics,
                                    const double* dev_q, double* dev_r, void* stream) {
    if (!grid || !numerics || !dev_q || !dev_r) return noalloc_fail(SFG_ERR_ARG, "null argument");
    const RecipeParts* rp = nullptr;
    for (const auto& p : kParts)
        if (p.id == numerics->recipe) rp = &p;
    if (!rp) return noalloc_fail(SFG_ERR_ARG, "convection recipe not provided on the GPU");
    if (numerics->precision != SFG_PREC_FP64 && numerics->precision != SFG_PREC_FP32_FLUX)
        return noalloc_fail(SFG_ERR_ARG, "unknown precision mode");
    if (!(numerics->gamma > 1.0) || !std::isfinite(numerics->gamma)) return noalloc_fail(SFG_ERR_ARG, "gamma must be > 1");
    if (grid->dim < 1 || grid->dim > 3) return noalloc_fail(SFG_ERR_ARG, "dim must be 1..3");
    const int reach = rp->scheme == WENO3 ? 2 : (rp->scheme == WENO7 ? 4 : 3);
    GridView g{};
    g.dim = grid->dim;
    long long nodes = 1;
    for (int a = 0; a < 3; ++a) {
        if (!(grid->h[a] > 0.0) || !std::isfinite(grid->h[a])) return noalloc_fail(SFG_ERR_ARG, "spacing must be > 0");
        g.n[a] = grid->n[a];
        if (a >= grid->dim) {
            if (grid->n[a] != 1) return noalloc_fail(SFG_ERR_ARG, "inactive axes must have 1 node");
            g.lo[a] = 0;
            g.hi[a] = 1;
            g.bc_lo[a] = g.bc_hi[a] = BC_TRANSMISSIVE;
            continue;
        }
        const bool plo = grid->bc_lo[a] == SFG_BC_PERIODIC, phi = grid->bc_hi[a] == SFG_BC_PERIODIC;
        if (plo != phi) return noalloc_fail(SFG_ERR_ARG, "periodic must be set on both ends of an axis");
        for (int b : {grid->bc_lo[a], grid->bc_hi[a]})
            if (b != SFG_BC_TRANSMISSIVE && b != SFG_BC_PERIODIC) return noalloc_fail(SFG_ERR_ARG, "unknown boundary kind");
        if (plo ? grid->n[a] < reach + 1 : grid->n[a] < 3) return noalloc_fail(SFG_ERR_ARG, "too few nodes on an axis");
        g.bc_lo[a] = grid->bc_lo[a];
        g.bc_hi[a] = grid->bc_hi[a];
        g.lo[a] = plo ? 0 : 1;
        g.hi[a] = plo ? grid->n[a] : grid->n[a] - 1;
        // each factor is at most the cap before it is multiplied in, so the
        // running product stays below cap^2 (< 2^37): no 64-bit overflow
        if (grid->n[a] > SFG_NOALLOC_MAX_NODES || nodes > SFG_NOALLOC_MAX_NODES) nodes = SFG_NOALLOC_MAX_NODES + 1LL;
        else nodes *= grid->n[a];
    }
    if (nodes > SFG_NOALLOC_MAX_NODES) {
        char msg[160];
        snprintf(msg, sizeof msg,
                 "grid of %lld x %lld x %lld nodes exceeds the fixed working array (SFG_NOALLOC_MAX_NODES = %d)",
                 (long long)grid->n[0], (long long)grid->n[1], (long long)grid->n[2], SFG_NOALLOC_MAX_NODES);
        return noalloc_fail(SFG_ERR_ARG, msg);
    }
    // uniform Cartesian metrics, formed exactly as sfg_create forms them
    const double hx = grid->h[0], hy = grid->h[1], hz = grid->h[2];
    g.jac = 1.0 / (hx * hy * hz);
    g.metric[0] = (hy * hz) * g.jac;
    g.metric[1] = (hx * hz) * g.jac;
    g.metric[2] = (hx * hy) * g.jac;
    for (int a = 0; a < 3; ++a) g.area[a] = 0.5 * (g.metric[a] / g.jac + g.metric[a] / g.jac);
    g.gamma = numerics->gamma;
    for (int a = 0; a < 3; ++a) g.h[a] = grid->h[a];
    g.cfl = numerics->cfl;
    g.vs = nodes;

    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // the call synchronises on `stream` and reads the status word back to
    // pageable host memory, neither of which a capturing stream allows
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone) {
        cudaGetLastError();
        return noalloc_fail(SFG_ERR_ARG, "sfg_residual_noalloc cannot run on a capturing stream");
    }
    double* base = nullptr;
    int rc = scratch_address(&base);
    if (rc) return rc;
    Clock* clock = reinterpret_cast<Clock*>(base);
    unsigned* flags = reinterpret_cast<unsigned*>(base + 16);
    double* r = base + kHeaderDoubles;
    const size_t rbytes = sizeof(double) * 5 * (size_t)nodes;

    // the array keeps the previous call's contents: clear what must start at 0
    cudaError_t e = cudaMemsetAsync(base, 0, kHeaderDoubles * sizeof(double), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(r, 0, rbytes, st);
    if (e != cudaSuccess) return noalloc_fail(SFG_ERR_CUDA, cudaGetErrorString(e));

    StageView sv{};
    sv.qs = dev_q;
    sv.q0 = dev_q;
    sv.r = r;
    sv.clock = clock;
    sv.flags = flags;
    sv.time_id = T_SSPRK3;
    for (int axis = 0; axis < grid->dim; ++axis) {
        sv.mode = (axis > 0 ? MODE_READ_R : 0) | (axis == grid->dim - 1 ? MODE_FINAL | MODE_RESIDUAL : 0);
        e = launch_sweep(rp->scheme, rp->flux, numerics->precision == SFG_PREC_FP64, axis, g, sv, st);
        if (e != cudaSuccess) return noalloc_fail(SFG_ERR_CUDA, cudaGetErrorString(e));
    }
    e = cudaMemcpyAsync(dev_r, r, rbytes, cudaMemcpyDeviceToDevice, st);
    unsigned host_flags = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&host_flags, flags, sizeof host_flags, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return noalloc_fail(SFG_ERR_CUDA, cudaGetErrorString(e));
    if (host_flags & FLAG_TENO_CUTOFF) return noalloc_fail(SFG_ERR_TENO_CUTOFF, "TENO5 rejected all sub-stencils");
    if (host_flags) return noalloc_fail(SFG_ERR_STATE, "invalid state on device");
    return SFG_OK;
}
