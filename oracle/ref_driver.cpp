// ref_driver.cpp -- drives the reference's own hot-path translation units.
//
// TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile against the sonicSolver
// sources where they lie (never copied into this repository) into
// oracle/_ref/libsfref.so.  It exposes the same flat C entry points as
// sf_oracle.h with the prefix sfr_, so the tests can pin the C restatement
// against the reference implementation on identical inputs.
//
// What runs reference code:
//   - the spatial operator: SF::divDispatch (solver/discretization/convection/
//     SF_div.h:212-243) with its WENO/TENO cores, characteristic matrices,
//     Steger-Warming / Rusanov / Lax-Friedrichs / Roe / Lax-Wendroff fluxes,
//     face loops and residual assembly, then
//     Math::spatialResidual (methods/numerics/structured/SF_residualAssembly.h:34-41);
//   - the CFL step: Numerics::RusanovEOS::deltaT (Flux/SF_rusanovEOS.cpp:110-147).
// What is restated here (the reference's versions need the full solver
// runtime): the ghost fill laws inside the time loop and the Euler /
// Shu-Osher SSPRK3 / RK4 stage arithmetic of
// solver/algorithm/time/SF_explicit.cpp:193-238,282-285.  The physical
// boundary laws themselves also run as reference code (sfr_fill_laws:
// Boundary::update, updateEnergyFromPressure) to pin the restatement.
#include "SF_field.h"
#include "SF_div.h"
#include "core/flux/SF_flux.h"
#include "core/residual/SF_residual.h"
#include "core/mesh/SF_dimension.h"
#include "methods/numerics/Flux/SF_rusanovEOS.h"
#include "methods/numerics/Flux/SF_sw.h"
#include "methods/numerics/Flux/SF_lxF.h"
#include "methods/numerics/Flux/SF_lw.h"
#include "methods/numerics/structured/SF_residualAssembly.h"
#include "models/physics/fluidStateModel/SF_singleFluidStateModel.h"
#include "models/physics/EOS/SF_perfectGasEOS.h"
#include "solver/boundary/SF_boundary.h"
#include "solver/boundary/SF_thermodynamicClosure.h"

#include "sf_oracle.h"

#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

// makeSingleFluidPerfectGas (fluidStateModel/SF_factory.h:21-33) without the
// multiphase headers that factory pulls in: inviscid (mu = 0), Pr = 0.72.
std::shared_ptr<const SF::Physics::FluidStateModel::SingleFluidStateModel> perfect_gas(double gamma) {
    const double gasConstant = 287.05, mu = 0.0, prandtl = 0.72;
    const double cp = gamma * gasConstant / (gamma - 1.0);
    return std::make_shared<const SF::Physics::FluidStateModel::SingleFluidStateModel>(
        std::make_shared<SF::Physics::EOS::PerfectGasEOS>(gamma, gasConstant), mu, mu * cp / prandtl);
}

struct RefCase {
    sfo_grid g;
    SF::Field field;
    SF::FluxField flux;
    SF::Residual residual;
    std::shared_ptr<const SF::Physics::FluidStateModel::SingleFluidStateModel> model;
};

int storage_extent(const sfo_grid* g, int d) { return g->n[d] + (d < g->dim ? 2 * g->ng : 0); }

// Build a reference Field (ghosts on every axis) with uniform Cartesian metrics.
void setup_case(RefCase& rc, const sfo_grid* g) {
    rc.g = *g;
    SF::Math::resetActiveDirections();
    for (int d = g->dim; d < 3; ++d) SF::Math::deactivateDirection(d);
    rc.field.setup(g->n[0], g->n[1], g->n[2], g->ng, 5);
    rc.model = perfect_gas(g->gamma);
    rc.field.setStateModel(rc.model);
    const double hx = g->h[0], hy = g->h[1], hz = g->h[2];
    const double J = hx * hy * hz;
    const double jac = 1.0 / J;
    for (int k = 0; k < rc.field.MZ(); ++k)
        for (int j = 0; j < rc.field.MY(); ++j)
            for (int i = 0; i < rc.field.MX(); ++i) {
                rc.field.Jac(i, j, k) = jac;
                rc.field.XiX(i, j, k) = (hy * hz) * jac;
                rc.field.XiY(i, j, k) = 0.0;
                rc.field.XiZ(i, j, k) = 0.0;
                rc.field.EtX(i, j, k) = 0.0;
                rc.field.EtY(i, j, k) = (hx * hz) * jac;
                rc.field.EtZ(i, j, k) = 0.0;
                rc.field.ZeX(i, j, k) = 0.0;
                rc.field.ZeY(i, j, k) = 0.0;
                rc.field.ZeZ(i, j, k) = (hx * hy) * jac;
                rc.field.X(i, j, k) = (i - g->ng) * hx;
                rc.field.Y(i, j, k) = (j - g->ng) * hy;
                rc.field.Z(i, j, k) = (k - g->ng) * hz;
            }
    // Curvilinear grids: the caller's per-node metrics (compact layout; the
    // Field's extra ghosts on inactive axes take the nearest compact point).
    if (g->metrics) {
        const int m0 = storage_extent(g, 0), m1 = storage_extent(g, 1), m2 = storage_extent(g, 2);
        int off[3];
        for (int d = 0; d < 3; ++d) off[d] = d < g->dim ? 0 : g->ng;
        for (int k = 0; k < rc.field.MZ(); ++k)
            for (int j = 0; j < rc.field.MY(); ++j)
                for (int i = 0; i < rc.field.MX(); ++i) {
                    int c[3] = {i - off[0], j - off[1], k - off[2]};
                    const int m[3] = {m0, m1, m2};
                    for (int d = 0; d < 3; ++d) c[d] = c[d] < 0 ? 0 : (c[d] >= m[d] ? m[d] - 1 : c[d]);
                    const double* src = g->metrics + (((long long)c[2] * m1 + c[1]) * m0 + c[0]) * 10;
                    rc.field.Jac(i, j, k) = src[0];
                    rc.field.XiX(i, j, k) = src[1];
                    rc.field.XiY(i, j, k) = src[2];
                    rc.field.XiZ(i, j, k) = src[3];
                    rc.field.EtX(i, j, k) = src[4];
                    rc.field.EtY(i, j, k) = src[5];
                    rc.field.EtZ(i, j, k) = src[6];
                    rc.field.ZeX(i, j, k) = src[7];
                    rc.field.ZeY(i, j, k) = src[8];
                    rc.field.ZeZ(i, j, k) = src[9];
                }
    }
    // Solver-boundary sets: the transmissive (zeroGradient) and LAW ends,
    // exactly the nodes that Boundary::Applicator marks
    // (SF_applicator.h:162-187).  Points are listed with the last axis
    // outermost, the order the restatement visits them in.
    std::map<std::string, std::vector<int>> sets;
    const int ng = g->ng;
    for (int d = 0; d < g->dim; ++d) {
        for (int end = 0; end < 2; ++end) {
            const int kind = end ? g->bc_hi[d] : g->bc_lo[d];
            if (kind != SFO_BC_TRANSMISSIVE && kind != SFO_BC_LAW) continue;
            std::string name = std::string("bc") + char('0' + d) + (end ? "hi" : "lo");
            auto& ids = sets[name];
            const int fixed = end ? g->n[d] - 1 + ng : ng;
            for (int k = 0; k < g->n[2]; ++k)
                for (int j = 0; j < g->n[1]; ++j)
                    for (int i = 0; i < g->n[0]; ++i) {
                        int idx[3] = {i + ng, j + ng, k + ng};
                        if (idx[d] != fixed) continue;
                        ids.push_back(rc.field.getIdx(idx[0], idx[1], idx[2]));
                    }
        }
    }
    rc.field.setBoundarySets(sets);
    rc.field.clearSolverBoundaryMask();
    for (auto& kv : sets) rc.field.markSolverBoundarySet(kv.first);
    const int mx = rc.field.MX(), my = rc.field.MY(), mz = rc.field.MZ();
    rc.flux.setup((size_t)3 * (size_t)mx * my * mz, 5);
    rc.residual.setup(mx, my, mz, 5);
}

// compact (ghosts on active axes only) <-> reference Field (ghosts everywhere)
void load_state(RefCase& rc, const double* Q) {
    const sfo_grid* g = &rc.g;
    const int m0 = storage_extent(g, 0), m1 = storage_extent(g, 1);
    int off[3];
    for (int d = 0; d < 3; ++d) off[d] = d < g->dim ? 0 : g->ng;
    for (int k = 0; k < rc.field.MZ(); ++k)
        for (int j = 0; j < rc.field.MY(); ++j)
            for (int i = 0; i < rc.field.MX(); ++i) {
                int c[3] = {i - off[0], j - off[1], k - off[2]};
                for (int d = 0; d < 3; ++d) {
                    const int m = storage_extent(g, d);
                    if (c[d] < 0) c[d] = 0;
                    if (c[d] >= m) c[d] = m - 1;
                }
                const double* q = Q + 5 * (((long long)c[2] * m1 + c[1]) * m0 + c[0]);
                for (int v = 0; v < 5; ++v) rc.field(i, j, k, v) = q[v];
            }
    rc.field.invalidateThermodynamicCache();
}

int scheme_of(int s, SF::FDM::ConvectionScheme* out) {
    switch (s) {
    case SFO_WENO3: *out = SF::FDM::ConvectionScheme::WENO3; return 0;
    case SFO_WENO5: *out = SF::FDM::ConvectionScheme::WENO5; return 0;
    case SFO_TENO5: *out = SF::FDM::ConvectionScheme::TENO5; return 0;
    case SFO_WENO7: *out = SF::FDM::ConvectionScheme::WENO7; return 0;
    }
    return SFO_ERR_ARG;
}

int flux_of(int f, SF::FDM::FluxSplitter* out) {
    switch (f) {
    case SFO_STEGER: *out = SF::FDM::FluxSplitter::StegerWarming; return 0;
    case SFO_RUSANOV: *out = SF::FDM::FluxSplitter::Rusanov; return 0;
    case SFO_LAXFRIEDRICHS: *out = SF::FDM::FluxSplitter::LaxFriedrichs; return 0;
    case SFO_ROE: *out = SF::FDM::FluxSplitter::Roe; return 0;
    case SFO_LAXWENDROFF: *out = SF::FDM::FluxSplitter::LaxWendroff; return 0;
    }
    return SFO_ERR_ARG;
}

}  // namespace

extern "C" {

// Residual of the reference spatial operator on Q (compact layout, ghosts
// already filled), written to R (compact layout; ghosts zero).
int sfr_rhs(const sfo_grid* g, int scheme, int flux, const double* Q, double* R) {
    try {
        SF::FDM::ConvectionScheme cs;
        SF::FDM::FluxSplitter fs;
        if (scheme_of(scheme, &cs) || flux_of(flux, &fs)) return SFO_ERR_ARG;
        RefCase rc;
        setup_case(rc, g);
        load_state(rc, Q);
        rc.flux.clear();
        rc.residual.clear();
        SF::divDispatch(rc.field, rc.flux, rc.residual, cs, fs, sfo_step_dt(),
                        SF::FDM::IBMBoundaryScheme::LowOrder, 0, g->gamma, *rc.model);
        const long long S = 5LL * storage_extent(g, 0) * storage_extent(g, 1) * storage_extent(g, 2);
        std::memset(R, 0, sizeof(double) * (size_t)S);
        const int m0 = storage_extent(g, 0), m1 = storage_extent(g, 1);
        int off[3];
        for (int d = 0; d < 3; ++d) off[d] = d < g->dim ? 0 : g->ng;
        const int ng = g->ng;
        for (int k = ng; k < ng + g->n[2]; ++k)
            for (int j = ng; j < ng + g->n[1]; ++j)
                for (int i = ng; i < ng + g->n[0]; ++i) {
                    const long long at = 5 * (((long long)(k - off[2]) * m1 + (j - off[1])) * m0 + (i - off[0]));
                    for (int v = 0; v < 5; ++v)
                        R[at + v] = SF::Math::spatialResidual(rc.field, rc.residual, i, j, k, v);
                }
        return SFO_OK;
    } catch (const std::exception&) {
        return SFO_ERR_STATE;
    }
}

int sfr_dt(const sfo_grid* g, const double* Q, double cfl, double* dt) {
    try {
        RefCase rc;
        setup_case(rc, g);
        load_state(rc, Q);
        *dt = SF::Numerics::RusanovEOS::deltaT(rc.field, *rc.model, cfl);
        return SFO_OK;
    } catch (const std::exception&) {
        return SFO_ERR_STATE;
    }
}

// ---- persistent case: Field allocated once, reference operator per stage ----

struct PersistentCase {
    RefCase rc;
    int scheme = 0, flux = 0;
    SF::FDM::ConvectionScheme cs{};
    SF::FDM::FluxSplitter fs{};
    std::vector<double> work;
};

static int case_rhs(void* ctx, const double* Q, double* R) {
    auto* pc = static_cast<PersistentCase*>(ctx);
    const sfo_grid* g = &pc->rc.g;
    try {
        load_state(pc->rc, Q);
        pc->rc.flux.clear();
        pc->rc.residual.clear();
        SF::divDispatch(pc->rc.field, pc->rc.flux, pc->rc.residual, pc->cs, pc->fs, sfo_step_dt(),
                        SF::FDM::IBMBoundaryScheme::LowOrder, 0, g->gamma, *pc->rc.model);
        const int m0 = storage_extent(g, 0), m1 = storage_extent(g, 1);
        int off[3];
        for (int d = 0; d < 3; ++d) off[d] = d < g->dim ? 0 : g->ng;
        const int ng = g->ng;
        for (int k = ng; k < ng + g->n[2]; ++k)
            for (int j = ng; j < ng + g->n[1]; ++j)
                for (int i = ng; i < ng + g->n[0]; ++i) {
                    const long long at =
                        5 * (((long long)(k - off[2]) * m1 + (j - off[1])) * m0 + (i - off[0]));
                    for (int v = 0; v < 5; ++v)
                        R[at + v] = SF::Math::spatialResidual(pc->rc.field, pc->rc.residual, i, j, k, v);
                }
        return SFO_OK;
    } catch (const std::exception&) {
        return SFO_ERR_STATE;
    }
}

static int case_dt(void* ctx, const double* Q, double cfl, double* dt) {
    auto* pc = static_cast<PersistentCase*>(ctx);
    try {
        load_state(pc->rc, Q);
        *dt = SF::Numerics::RusanovEOS::deltaT(pc->rc.field, *pc->rc.model, cfl);
        return SFO_OK;
    } catch (const std::exception&) {
        return SFO_ERR_STATE;
    }
}

void* sfr_case_create(const sfo_grid* g, int scheme, int flux) {
    auto* pc = new PersistentCase;
    if (scheme_of(scheme, &pc->cs) || flux_of(flux, &pc->fs)) {
        delete pc;
        return nullptr;
    }
    pc->scheme = scheme;
    pc->flux = flux;
    setup_case(pc->rc, g);
    pc->work.assign((size_t)5 * 5 * storage_extent(g, 0) * storage_extent(g, 1) * storage_extent(g, 2), 0.0);
    return pc;
}

void sfr_case_destroy(void* h) { delete static_cast<PersistentCase*>(h); }

int sfr_case_rhs(void* h, const double* Q, double* R) { return case_rhs(h, Q, R); }

int sfr_case_dt(void* h, const double* Q, double cfl, double* dt) { return case_dt(h, Q, cfl, dt); }

// One full explicit step of size dt (ghost fill and stage arithmetic restated,
// spatial operator from the reference).
int sfr_case_step(void* h, int time_id, double* Q, double dt) {
    auto* pc = static_cast<PersistentCase*>(h);
    const int ns = time_id == SFO_EULER ? 1 : (time_id == SFO_SSPRK3 ? 3 : (time_id == SFO_RK4 ? 4 : 0));
    if (!ns) return SFO_ERR_ARG;
    int prep = sfo_fill_ghosts(&pc->rc.g, Q);  // FlowStepPrepare
    if (prep) return prep;
    for (int s = 0; s < ns; ++s) {
        int err = sfo_stage_fn(&pc->rc.g, case_rhs, pc, time_id, Q, dt, s, pc->work.data());
        if (err) return err;
    }
    return SFO_OK;
}

int sfr_case_advance(void* h, int time_id, double* Q, double t_start, double t_end, double cfl,
                     double max_dt, double write_interval, int max_steps, double* dt_out,
                     int* steps_done, double* t_final) {
    auto* pc = static_cast<PersistentCase*>(h);
    return sfo_advance_fn(&pc->rc.g, case_rhs, case_dt, pc, time_id, Q, t_start, t_end, cfl, max_dt,
                          write_interval, max_steps, dt_out, steps_done, t_final);
}

// The reference's own physical boundary laws on Q (compact layout): the
// density, velocity and pressure settings of every LAW end, applied as
// Boundary::Applicator::apply does (SF_applicator.h:51-83) between the cache
// invalidations of the conservative RHS (SF_conservativeRHS.cpp:91-95).
// Settings are listed x low, x high, y low, ... (the restatement's order).
int sfr_fill_laws(const sfo_grid* g, double* Q) {
    try {
        RefCase rc;
        setup_case(rc, g);
        load_state(rc, Q);
        std::vector<SF::BCSetting<double>> density, pressure;
        std::vector<SF::BCSetting<SF::Vector3>> velocity;
        auto type_of = [](int law) {
            return law == SFO_LAW_FIXED_VALUE ? SF::FIXED_VALUE
                   : law == SFO_LAW_SYMMETRY  ? SF::SYMMETRY
                                              : SF::ZERO_GRADIENT;
        };
        for (int d = 0; d < g->dim; ++d)
            for (int end = 0; end < 2; ++end) {
                if ((end ? g->bc_hi[d] : g->bc_lo[d]) != SFO_BC_LAW) continue;
                const sfo_law& law = g->law[2 * d + end];
                const std::string name = std::string("bc") + char('0' + d) + (end ? "hi" : "lo");
                density.push_back({name, type_of(law.rho), law.rho_value});
                velocity.push_back({name, type_of(law.U), SF::Vector3(law.U_value[0], law.U_value[1], law.U_value[2])});
                pressure.push_back({name, type_of(law.p), law.p_value});
            }
        rc.field.invalidateThermodynamicCache();
        SF::Boundary::update<double>(rc.field, density, SF::RHO);
        SF::Boundary::update<SF::Vector3>(rc.field, velocity, SF::RU);
        SF::Boundary::updateEnergyFromPressure(rc.field, pressure);
        rc.field.invalidateThermodynamicCache();
        // reference Field -> compact layout (every compact storage position)
        const int m0 = storage_extent(g, 0), m1 = storage_extent(g, 1), m2 = storage_extent(g, 2);
        int off[3];
        for (int d = 0; d < 3; ++d) off[d] = d < g->dim ? 0 : g->ng;
        for (int k = 0; k < m2; ++k)
            for (int j = 0; j < m1; ++j)
                for (int i = 0; i < m0; ++i) {
                    double* q = Q + 5 * (((long long)k * m1 + j) * m0 + i);
                    for (int v = 0; v < 5; ++v) q[v] = rc.field(i + off[0], j + off[1], k + off[2], v);
                }
        return SFO_OK;
    } catch (const std::exception&) {
        return SFO_ERR_STATE;
    }
}

// Scalar cores and fluxes straight from the reference (known-answer tests).
double sfr_weno5_core(const double* v) { return SF::WENO5::weno5_core(v); }
double sfr_teno5_core(const double* v) { return SF::TENO5::teno5_core(v); }
double sfr_weno3_core(const double* v) { return SF::WENO3::weno3_core(v); }
double sfr_weno7_core(const double* v) { return SF::WENO7::weno7_core(v); }
void sfr_char_matrix(const double* q, const double* n, double gamma, double* L, double* R) {
    SF::Riemann::buildCharacteristicMatrix(q, n, gamma, L, R);
}
int sfr_rusanov_flux(const double* qL, const double* qR, const double* n, double gamma, double* out) {
    try {
        auto model = perfect_gas(gamma);
        SF::Numerics::RusanovEOS::faceFlux(*model, qL, qR, {n[0], n[1], n[2]}, out, 5);
        return SFO_OK;
    } catch (const std::exception&) {
        return SFO_ERR_STATE;
    }
}
void sfr_roe_flux(const double* qL, const double* qR, const double* n, double gamma, double* out) {
    SF::Flux::RoeFlux::flux(qL, qR, n, out, gamma);
}
// The reference's Steger-Warming, Lax-Friedrichs and Lax-Wendroff face
// fluxes (Flux/SF_sw.cpp, SF_lxF.cpp, SF_lw.cpp).  They exit the process on an
// invalid state, so callers pass valid states only.
void sfr_steger_flux(const double* qL, const double* qR, const double* n, double gamma, double* out) {
    SF::Flux::StegerWarmingFlux::flux(qL, qR, n, out, gamma);
}
void sfr_lf_flux(const double* qL, const double* qR, const double* n, double gamma, double* out) {
    SF::Flux::LaxFriedrichsFlux::flux(qL, qR, n, out, gamma);
}
void sfr_lw_flux(const double* qL, const double* qR, const double* n, double dt, double spacing, double gamma,
                 double* out) {
    SF::Flux::LaxWendroffFlux::flux(qL, qR, n, dt, spacing, out, gamma);
}

}  // extern "C"
