// sfh_case.hpp -- a sonicSolver case directory, read into what the explicit
// Euler provider needs.
//
// Files (located through the case's registries, as the reference does):
//   solvers/solvers.yaml -> runtime (startTime, endTime, CFL, writeControl,
//     writeInterval, writeInitial, output.jobName / outputDir, maxDeltaT),
//     numerics (time.default, terms.convection), algorithm (type);
//   models/models.yaml -> thermoDynamics (perfectGas gamma, R, transport
//     mu), and the switches of the IBM, MRF, turbulence, multiPhase,
//     phaseChange and thermophysical modules (gravity and geometry entries
//     are inert on the density-based path);
//   solvers/solvers.yaml -> equations (preset), ILW (enabled);
//   mesh/mesh.yaml -> generation (JSON: vertices, blocks[0].vertices /
//     cells / grading, scale, nGhost, arc edges; one block: an axis-aligned
//     box runs on the uniform Cartesian path, a graded or curved block with
//     the generator's node coordinates and metrics, sfh_mesh.hpp);
//   fields/fields.yaml -> internalField (rho, U, p: uniform / default plus
//     the mesh sets leftHalf, rightHalf, all) and boundaries (per variable,
//     per patch: fixedValue, zeroGradient, symmetry, velocity noSlip / slip,
//     empty, none (frozen ghosts), and this provider's periodic).
// Mesh sets follow the structured generator
// (src/infrastructure/mesh/createMesh/SF_meshGen.cpp:514-541): patches Left /
// Right (i = 0 / nx-1), sideWalls (j ends), frontBack (k ends); leftHalf holds
// the nodes with i < nx/2, rightHalf the rest.
#pragma once

#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/sonicsolver_b200.h"
#include "sfh_mesh.hpp"

namespace sfh {

// A case the provider cannot run; the message says what and why.
struct Unsupported : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// One field's condition at one patch (compactBoundary,
// src/infrastructure/io/case/SF_case.cpp:22-29): the law token as written
// and its value (fixedValue: 1 number for rho and p, 3 for U).
struct FieldCondition {
    std::string type;
    std::vector<double> value;
};

struct InitialValue {
    std::vector<double> base;                                       // uniform / default
    std::vector<std::pair<std::string, std::vector<double>>> sets;  // named sets, file order
};

struct CaseSpec {
    std::string dir, name;
    // mesh
    double lo[3] = {0, 0, 0}, hi[3] = {1, 1, 1};
    int cells[3] = {1, 1, 1};
    int ghost_layers = 3;
    MeshGeneration mesh;       // the block as generated
    bool curvilinear = false;  // not a uniform axis-aligned box: metrics from `mesh`
    // physics
    double gamma = 1.4, gas_R = 287.05;
    // numerics
    std::string convection, time_recipe, algorithm;
    double max_dt = 0.0;
    // runtime
    double start_time = 0.0, end_time = 0.0, cfl = 0.5, write_interval = 0.0;
    bool write_initial = false;
    std::string write_control = "runTime", output_dir = "result", job_name;
    // patch -> field ("rho", "U", "p") -> condition
    std::map<std::string, std::map<std::string, FieldCondition>> patch_bc;
    // field ("rho", "U", "p") -> its patches in file order (the order the
    // reference's writer numbers boundary sets in)
    std::map<std::string, std::vector<std::string>> bc_order;
    // fields declared in the fields registry (fields/fields.yaml), file order
    struct DeclaredField {
        std::string name, output_name;
        bool output = true;
    };
    std::vector<DeclaredField> declared_fields;
    InitialValue rho, U, p;
    // enabled physics outside the inviscid single-fluid Euler equations (an
    // immersed boundary, MRF, a turbulence model, multiphase, phase change, a
    // temperature equation, viscous transport, ILW, a non-compressible
    // equation preset), one reason each; build_grid refuses a case with any
    std::vector<std::string> unsupported_physics;
};

CaseSpec load_case(const std::string& dir);

// The provider's grid and initial state for a case.
struct GridSetup {
    sfg_grid_desc grid{};
    sfg_boundary_law laws[6] = {};  // [2 * axis + end] of SFG_BC_LAW ends
    int nodes[3] = {1, 1, 1};
    double origin[3] = {0, 0, 0};
    std::vector<double> q;  // AoS [k][j][i][v] over the nodes, conserved
};

// An active patch with no condition becomes SFG_BC_FROZEN (the reference
// keeps the initial ghost state there and advances the boundary node).
// A patch whose rho, U and p are all zeroGradient is SFG_BC_TRANSMISSIVE;
// one with fixedValue or symmetry laws is SFG_BC_LAW with those laws.
// Throws Unsupported for what this provider does not run (an algorithm other
// than densityBase; enabled physics listed in unsupported_physics; periodic
// ends on a graded or curved block; a patch with conditions for only some of
// rho, U, p).
GridSetup build_grid(const CaseSpec& c);

}  // namespace sfh
