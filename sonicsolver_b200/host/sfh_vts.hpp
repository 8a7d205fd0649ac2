// sfh_vts.hpp -- ASCII VTK StructuredGrid (.vts) output of a node state, in
// the reference's result layout (ResultWriter::writeToDisk,
// src/infrastructure/io/SF_vtkStructuredWriter.cpp:22-207, with the output
// fields of ModelLoader::configureOutput, src/app/application/model/
// SF_output.cpp:8-118):
//   * one piece over the reference Field's nodes: cells + 1 per axis, so an
//     axis the provider does not solve (an empty patch pair) is written as
//     its node planes with the same state on each; a periodic axis keeps the
//     provider's nodes;
//   * Points, then PointData: the Int32 boundary-set arrays BC_ID,
//     BC_ID_rho, BC_ID_U, BC_ID_p (0 inside; k + 1 on the nodes of the k-th
//     set a boundary condition names, sets numbered by first appearance over
//     the rho, U, p conditions in file order, later sets winning on shared
//     nodes; BC_ID takes the U, then the p number where set) with their
//     legend comment, then the fluid arrays Density, Velocity (3 components)
//     and Pressure -- renamed or dropped as the case's fields registry
//     declares them (rho / U / p with output true take those names) -- in
//     name order;
//   * Float64 values with 17 significant digits.
#pragma once

#include <string>
#include <vector>

#include "sfh_case.hpp"

namespace sfh {

enum class VtsQuantity { Density, Velocity, Pressure };

struct VtsArray {
    std::string name;
    VtsQuantity what;
};

struct VtsLayout {
    int nodes[3] = {1, 1, 1};      // the provider's nodes per axis (the state's layout)
    int out_nodes[3] = {1, 1, 1};  // nodes written per axis
    double origin[3] = {0, 0, 0};  // coordinate of written node (0, 0, 0)
    double h[3] = {1, 1, 1};       // spacing of the written nodes (a box)
    // x, y, z per written node (x fastest) of a graded or curved block; empty:
    // origin + (i, j, k) h
    std::vector<double> points;
    std::vector<int> bc_id[4];     // BC_ID, BC_ID_rho, BC_ID_U, BC_ID_p per written node
    std::string legend;            // names of the numbered sets, "1=Left, 2=Right, ..."
    std::vector<VtsArray> arrays;  // fluid arrays in write order
};

// The output layout of a case.  `block_points`: the generated coordinates of
// a graded or curved block over all (cells + 1)^3 nodes, or empty.
VtsLayout vts_layout(const CaseSpec& c, const GridSetup& g, const std::vector<double>& block_points);

// q: conserved AoS [k][j][i][v] over the provider's nodes.  Returns false
// when the file cannot be written.
bool write_vts(const std::string& path, const VtsLayout& geo, const std::vector<double>& q, double gamma);

}  // namespace sfh
