// sfh_mesh.hpp -- node coordinates and Field metrics of a generated
// structured block (mesh/generation.yaml), for blocks that are not a uniform
// axis-aligned box: graded blocks and blocks with arc edges.
//
// This is the geometry the reference builds before a run:
//   * node coordinates: trilinear interpolation of the 8 block vertices with
//     the per-axis grading (MeshGen::generateBlockPoints,
//     src/infrastructure/mesh/createMesh/SF_meshGen.cpp:34-76), or, when the
//     generation lists edges, transfinite interpolation over the 12 block
//     edges with arcs through a point (generateTFIBlock, SF_meshGen.cpp:797-918;
//     arcGeometry / arcPoint / edgeEval, SF_edges.h:78-176);
//   * the Field's ghost coordinates, extrapolated linearly axis by axis
//     (Mesh::generateGhostCells / extrapolateCoord,
//     src/infrastructure/mesh/SF_mesh.cpp:491-586);
//   * metrics per Field point: the symmetric conservative (Thomas-Lombard)
//     cofactors and J = (r_xi . c_xi + r_eta . c_eta + r_zeta . c_zeta) / 3 on
//     every point one layer in, the outermost layer copied from its inner
//     neighbour (Mesh::computeMetrics / applyBoundaryMetrics,
//     SF_mesh.cpp:219-345,439-474);
//   * the discrete metric identity the reference audits before a run
//     (Mesh::auditMetricIdentity, SF_mesh.cpp:348-437).
// The same operations in the same order, so the metrics are the reference's
// own to the last bit; they reach the provider through sfg_set_metrics
// (Field layout).
#pragma once

#include <array>
#include <string>
#include <vector>

namespace sfh {

struct ArcEdge {
    int v0 = 0, v1 = 0;                 // vertex indices of the generation
    std::array<double, 3> point{};      // a point the arc passes through
};

struct MeshGeneration {
    double scale = 1.0;
    int n_ghost = 3;
    std::vector<std::array<double, 3>> vertices;
    int verts[8] = {0, 1, 2, 3, 4, 5, 6, 7};  // the block's hex, reference vertex order
    int cells[3] = {1, 1, 1};
    double grading[3] = {1.0, 1.0, 1.0};
    std::vector<ArcEdge> edges;         // every edge of the generation file

    // An axis-aligned box listed in the canonical corner order, with unit
    // grading and no edges: the provider's uniform Cartesian path needs no
    // metrics there.
    bool uniform_box() const;
};

// Node coordinates of the block: (cells + 1) points per axis, x fastest.
void block_points(const MeshGeneration& m, std::vector<double>& x, std::vector<double>& y, std::vector<double>& z);

// The reference Field's geometry: (cells + 1 + 2 ng) points per axis, ng
// ghost layers on every axis, x fastest.
struct FieldGeometry {
    int ext[3] = {0, 0, 0};
    int ng = 0;
    std::vector<double> x, y, z;        // coordinates per point
    std::vector<double> metrics;        // per point: Jac = 1/J, XiX, XiY, XiZ, EtX, ..., ZeZ
    double identity_residual = 0.0;     // max |sum_d (C_d(i) - C_d(i-1))| over the nodes
    double identity_tolerance = 0.0;    // 65536 eps max |C|: the reference's bar
    long long at(int i, int j, int k) const { return ((long long)k * ext[1] + j) * ext[0] + i; }
};

// Builds the Field geometry.  `active` marks the solved axes (the metric
// identity is audited over those, as the reference does).  Throws
// std::runtime_error on a degenerate Jacobian (the reference exits there).
FieldGeometry field_geometry(const MeshGeneration& m, int ng, const bool active[3]);

}  // namespace sfh
