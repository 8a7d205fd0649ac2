// sfh_case.hpp -- a sonicSolver case directory, read into what the explicit
// Euler provider needs.
//
// Files (located through the case's registries, as the reference does):
//   solvers/solvers.yaml -> runtime (startTime, endTime, CFL, writeControl,
//     writeInterval, writeInitial, output.jobName / outputDir, maxDeltaT),
//     numerics (time.default, terms.convection), algorithm (type);
//   models/models.yaml -> thermoDynamics (perfectGas gamma, R);
//   mesh/mesh.yaml -> generation (JSON: vertices, blocks[0].cells, scale,
//     nGhost; one axis-aligned box block);
//   fields/fields.yaml -> internalField (rho, U, p: uniform / default plus
//     the mesh sets leftHalf, rightHalf, all) and boundaries (per variable,
//     per patch: zeroGradient, empty, none (frozen ghosts), and this
//     provider's periodic).
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

namespace sfh {

// A case the provider cannot run; the message says what and why.
struct Unsupported : std::runtime_error {
    using std::runtime_error::runtime_error;
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
    // physics
    double gamma = 1.4, gas_R = 287.05;
    // numerics
    std::string convection, time_recipe, algorithm;
    double max_dt = 0.0;
    // runtime
    double start_time = 0.0, end_time = 0.0, cfl = 0.5, write_interval = 0.0;
    bool write_initial = false;
    std::string write_control = "runTime", output_dir = "result", job_name;
    // one condition per patch (rho, U and p must agree)
    std::map<std::string, std::string> patch_bc;
    InitialValue rho, U, p;
};

CaseSpec load_case(const std::string& dir);

// The provider's grid and initial state for a case.
struct GridSetup {
    sfg_grid_desc grid{};
    int nodes[3] = {1, 1, 1};
    double origin[3] = {0, 0, 0};
    std::vector<double> q;  // AoS [k][j][i][v] over the nodes, conserved
};

// An active patch with no condition becomes SFG_BC_FROZEN (the reference
// keeps the initial ghost state there and advances the boundary node).
// Throws Unsupported for what this provider does not run (curvilinear or
// graded blocks; conditions other than zeroGradient, periodic and empty).
GridSetup build_grid(const CaseSpec& c);

}  // namespace sfh
