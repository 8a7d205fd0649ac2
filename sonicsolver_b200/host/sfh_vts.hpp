// sfh_vts.hpp -- ASCII VTK StructuredGrid (.vts) output of a node state.
//
// Same file kind as the reference's structured writer
// (src/infrastructure/io/SF_vtkStructuredWriter.cpp:32,114-170): one piece
// over the nodes (no ghosts), node coordinates as Points, and Float64 point
// data rho, U (3 components), p and E written with 17 significant digits, so
// a file read back gives the state to the last bit.
#pragma once

#include <string>
#include <vector>

namespace sfh {

struct VtsGeometry {
    int nodes[3];       // nodes per axis (1 on inactive axes)
    double origin[3];   // coordinate of node (0, 0, 0)
    double h[3];        // node spacing (unused on inactive axes)
    // node coordinates x, y, z per node (x fastest) of a graded or curved
    // block; null: origin + (i, j, k) h
    const std::vector<double>* points = nullptr;
};

// q: conserved AoS [k][j][i][v] over the nodes.  Returns false when the file
// cannot be written.
bool write_vts(const std::string& path, const VtsGeometry& geo, const std::vector<double>& q, double gamma,
               double time);

}  // namespace sfh
