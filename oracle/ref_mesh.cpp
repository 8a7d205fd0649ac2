// ref_mesh.cpp -- test infrastructure: a C entry over the reference's own
// structured-block generator (MeshGen::generateStructuredMesh,
// src/infrastructure/mesh/createMesh/SF_meshGen.cpp:77-110, compiled where
// it lies), so that the tests can check the host's restatement of it
// (sonicsolver_b200/host/sfh_mesh.cpp) bit for bit.  Never part of the
// product.
#include <cstring>
#include <vector>

#include "SF_meshGen.h"

extern "C" {

// One block: vertices (n_vertices x 3) and scale as the generation file
// holds them, the block's hex (8 vertex indices), cells and grading, arc
// edges (n_edges pairs of vertex indices and their points).  Writes
// (cells + 1) points per axis to xyz (x, y, z per point, x fastest).
// Returns 0, or 1 on a bad argument.
int sfr_mesh_points(int n_vertices, const double* vertices, double scale, const int* hex, const int* cells,
                    const double* grading, int n_edges, const int* edge_ends, const double* edge_points,
                    double* xyz) {
    if (n_vertices < 1 || !vertices || !hex || !cells || !grading || !xyz || n_edges < 0) return 1;
    SF::MeshParameters p;
    p.scale = scale;
    for (int v = 0; v < n_vertices; ++v) p.vertices.push_back({vertices[3 * v], vertices[3 * v + 1], vertices[3 * v + 2]});
    SF::MeshBlock b;
    for (int c = 0; c < 8; ++c) {
        if (hex[c] < 0 || hex[c] >= n_vertices) return 1;
        b.verts[c] = hex[c];
    }
    for (int d = 0; d < 3; ++d) {
        if (cells[d] < 1) return 1;
        b.cells[d] = cells[d];
        b.grade[d] = grading[d];
    }
    p.blocks.push_back(b);
    for (int e = 0; e < n_edges; ++e) {
        SF::MeshEdge m;
        m.type = SF::EdgeType::ARC;
        m.v0 = edge_ends[2 * e];
        m.v1 = edge_ends[2 * e + 1];
        m.arcP = {edge_points[3 * e], edge_points[3 * e + 1], edge_points[3 * e + 2]};
        p.edges.push_back(m);
    }
    std::vector<double> x, y, z;
    std::vector<int> sizes;
    SF::MeshGen::generateStructuredMesh(p, x, y, z, sizes);
    for (size_t i = 0; i < x.size(); ++i) {
        xyz[3 * i] = x[i];
        xyz[3 * i + 1] = y[i];
        xyz[3 * i + 2] = z[i];
    }
    return 0;
}

}  // extern "C"
