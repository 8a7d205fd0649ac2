// sfh_mesh.cpp -- generated block coordinates and the reference Field's
// metrics (see sfh_mesh.hpp).  Every sum and product below is evaluated in
// the order the reference writes it, so that coordinates and metrics agree
// to the last bit with the reference's own (the host build does not
// contract multiply-adds).
#include "sfh_mesh.hpp"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <stdexcept>
#include <string>

namespace sfh {

namespace {

struct V3 {
    double x, y, z;
};
V3 v3(const std::array<double, 3>& a) { return {a[0], a[1], a[2]}; }
V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V3 mul(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
double norm(V3 a) { return std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
// divides each component (the reference divides, it does not multiply by
// the reciprocal)
V3 divide(V3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }

struct Arc {
    V3 center{0, 0, 0};
    double radius = 0, angle = 0;
    V3 start{1, 0, 0}, bitangent{0, 1, 0};
};

// The circle through v0, mid and v1 and the arc from v0 to v1 that passes
// mid (arcGeometry, SF_edges.h:77-160).  Centre: the intersection of the
// perpendicular bisectors of v0-v1 and v0-mid in the circle's plane, solved
// in the first coordinate plane whose determinant is not small (the step
// size t1 keeps the reference's choice of formula).  Angle: the short arc
// when mid lies on it, else the long one; the axis is turned so that the
// arc runs from v0 towards v1 through mid.
Arc arc_geometry(V3 v0, V3 v1, V3 mid) {
    Arc g;
    V3 axis = cross(sub(v1, v0), sub(mid, v0));
    const double len = norm(axis);
    if (len < 1e-20) {  // collinear: a point arc at v0
        g.center = v0;
        return g;
    }
    axis = divide(axis, len);
    const V3 mAB = mul(add(v0, v1), 0.5), mAC = mul(add(v0, mid), 0.5);
    const V3 nAB = cross(axis, sub(v1, v0)), nAC = cross(axis, sub(mid, v0));
    const double det_yz = nAB.y * nAC.z - nAB.z * nAC.y;
    double det = det_yz;
    if (std::fabs(det) < 1e-12) det = nAB.x * nAC.z - nAB.z * nAC.x;
    if (std::fabs(det) < 1e-12) det = nAB.x * nAC.y - nAB.y * nAC.x;
    double t1 = 0.0;
    if (std::fabs(det) > 1e-20) {
        const double dx = mAC.x - mAB.x, dy = mAC.y - mAB.y, dz = mAC.z - mAB.z;
        if (std::fabs(det_yz) > 1e-12)
            t1 = (dy * nAC.z - dz * nAC.y) / det;
        else
            t1 = (dx * nAC.y - dy * nAC.x) / (det + 1e-20);
    }
    g.center = {mAB.x + t1 * nAB.x, mAB.y + t1 * nAB.y, mAB.z + t1 * nAB.z};
    V3 start = sub(v0, g.center);
    g.radius = norm(start);
    if (g.radius < 1e-20) return g;  // start / bitangent keep their defaults
    start = divide(start, g.radius);
    const V3 e = sub(v1, g.center);
    const V3 end = divide(e, norm(e) + 1e-20);
    const double c = std::min(1.0, std::max(-1.0, dot(start, end)));
    const double short_angle = std::acos(c);
    const double sign_end = dot(cross(start, end), axis);
    const V3 r_mid = sub(mid, g.center);
    const V3 mid_dir = divide(r_mid, norm(r_mid) + 1e-20);
    const double sign_mid = dot(cross(start, mid_dir), axis);
    if (sign_end * sign_mid >= 0) {  // mid on the short arc
        g.angle = short_angle;
        if (sign_end < 0) axis = {-axis.x, -axis.y, -axis.z};
    } else {
        g.angle = 2.0 * M_PI - short_angle;
        if (sign_mid < 0) axis = {-axis.x, -axis.y, -axis.z};
    }
    g.start = start;
    g.bitangent = cross(axis, start);
    return g;
}

// Point at parameter t of an edge (edgeEval / arcEval / arcPoint,
// SF_edges.h:162-175): centre + R (cos th start + sin th bitangent) with
// th = t angle on an arc (the arc's point scaled like the vertices),
// v0 + t (v1 - v0) on a line.
V3 edge_point(V3 v0, V3 v1, const ArcEdge* arc, double scale, double t) {
    if (arc) {
        const Arc g = arc_geometry(v0, v1, mul(v3(arc->point), scale));
        const double th = t * g.angle;
        const double c = std::cos(th), s = std::sin(th);
        return {g.center.x + g.radius * (c * g.start.x + s * g.bitangent.x),
                g.center.y + g.radius * (c * g.start.y + s * g.bitangent.y),
                g.center.z + g.radius * (c * g.start.z + s * g.bitangent.z)};
    }
    return {v0.x + t * (v1.x - v0.x), v0.y + t * (v1.y - v0.y), v0.z + t * (v1.z - v0.z)};
}

// Parameter of point i of n along an axis with grading g (paramCoord,
// SF_meshGen.cpp:44-49): cell sizes change by the factor g from cell to cell.
double graded(int i, int n, double g) {
    if (n <= 1) return 0.0;
    if (g == 1.0) return (double)i / (n - 1);
    const double r = (g == 0.0) ? 1.0 : g;
    return (1.0 - std::pow(r, i)) / (1.0 - std::pow(r, n - 1));
}

double comp(const V3& v, int c) { return c == 0 ? v.x : (c == 1 ? v.y : v.z); }

}  // namespace

bool MeshGeneration::uniform_box() const {
    if (!edges.empty()) return false;  // any edge sends the generator to TFI
    for (double g : grading)
        if (g != 1.0) return false;
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int c = 0; c < 8; ++c)
        for (int d = 0; d < 3; ++d) {
            lo[d] = std::min(lo[d], vertices[verts[c]][d] * scale);
            hi[d] = std::max(hi[d], vertices[verts[c]][d] * scale);
        }
    // hex corner c at (i, j, k) = (0,0,0), (1,0,0), (1,1,0), (0,1,0), then
    // the same at k = 1: each must sit on that corner of the box, so that
    // node (i, j, k) is lo + (i hx, j hy, k hz)
    static const int corner[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                                     {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
    for (int c = 0; c < 8; ++c)
        for (int d = 0; d < 3; ++d) {
            const double x = vertices[verts[c]][d] * scale;
            const double want = corner[c][d] ? hi[d] : lo[d];
            if (std::fabs(x - want) > 1e-12 * (1 + std::fabs(want))) return false;
        }
    return true;
}

void block_points(const MeshGeneration& m, std::vector<double>& x, std::vector<double>& y, std::vector<double>& z) {
    const int np[3] = {m.cells[0] + 1, m.cells[1] + 1, m.cells[2] + 1};
    const size_t total = (size_t)np[0] * np[1] * np[2];
    x.resize(total);
    y.resize(total);
    z.resize(total);
    V3 V[8];
    for (int c = 0; c < 8; ++c) {
        const auto& v = m.vertices[m.verts[c]];
        V[c] = {v[0] * m.scale, v[1] * m.scale, v[2] * m.scale};
    }
    size_t idx = 0;
    if (m.edges.empty()) {
        // trilinear interpolation with grading (generateBlockPoints,
        // SF_meshGen.cpp:34-76): corner (ii, jj, kk) is hex vertex
        // corner_of[kk][jj][ii], summed kk, jj, ii outermost to innermost
        static const int corner_of[2][2][2] = {{{0, 1}, {3, 2}}, {{4, 5}, {7, 6}}};
        for (int k = 0; k < np[2]; ++k) {
            const double zeta = graded(k, np[2], m.grading[2]);
            for (int j = 0; j < np[1]; ++j) {
                const double eta = graded(j, np[1], m.grading[1]);
                for (int i = 0; i < np[0]; ++i, ++idx) {
                    const double xi = graded(i, np[0], m.grading[0]);
                    const double s[3] = {xi, eta, zeta};
                    double p[3] = {0.0, 0.0, 0.0};
                    for (int kk = 0; kk < 2; ++kk)
                        for (int jj = 0; jj < 2; ++jj)
                            for (int ii = 0; ii < 2; ++ii) {
                                const double w = (ii ? s[0] : 1.0 - s[0]) * (jj ? s[1] : 1.0 - s[1]) *
                                                 (kk ? s[2] : 1.0 - s[2]);
                                const V3& v = V[corner_of[kk][jj][ii]];
                                p[0] += w * v.x;
                                p[1] += w * v.y;
                                p[2] += w * v.z;
                            }
                    x[idx] = p[0];
                    y[idx] = p[1];
                    z[idx] = p[2];
                }
            }
        }
        return;
    }
    // transfinite interpolation over the 12 edges (generateTFIBlock,
    // SF_meshGen.cpp:797-918, with the edge table of buildEdgeTable,
    // :772-795): xi-edges 0-1, 3-2, 4-5, 7-6; eta-edges 0-3, 1-2, 4-7, 5-6;
    // zeta-edges 0-4, 1-5, 3-7, 2-6 (hex corners).  An edge of the generation
    // joining the same two vertices, in either direction, makes it an arc.
    // The parameters are uniform: the generator's TFI path takes no grading.
    static const int ends[12][2] = {{0, 1}, {3, 2}, {4, 5}, {7, 6}, {0, 3}, {1, 2},
                                    {4, 7}, {5, 6}, {0, 4}, {1, 5}, {3, 7}, {2, 6}};
    const ArcEdge* arc[12];
    for (int e = 0; e < 12; ++e) {
        arc[e] = nullptr;
        const int a = m.verts[ends[e][0]], b = m.verts[ends[e][1]];
        for (const auto& ed : m.edges)
            if ((ed.v0 == a && ed.v1 == b) || (ed.v0 == b && ed.v1 == a)) {
                arc[e] = &ed;
                break;
            }
    }
    auto E = [&](int e, double t) { return edge_point(V[ends[e][0]], V[ends[e][1]], arc[e], m.scale, t); };
    for (int k = 0; k < np[2]; ++k) {
        const double zeta = (np[2] > 1) ? (double)k / (np[2] - 1) : 0.0;
        for (int j = 0; j < np[1]; ++j) {
            const double eta = (np[1] > 1) ? (double)j / (np[1] - 1) : 0.0;
            for (int i = 0; i < np[0]; ++i, ++idx) {
                const double xi = (np[0] > 1) ? (double)i / (np[0] - 1) : 0.0;
                const V3 ex[4] = {E(0, xi), E(1, xi), E(2, xi), E(3, xi)};
                const V3 ee[4] = {E(4, eta), E(5, eta), E(6, eta), E(7, eta)};
                const V3 ez[4] = {E(8, zeta), E(9, zeta), E(10, zeta), E(11, zeta)};
                double p[3];
                for (int c = 0; c < 3; ++c) {
                    double v = 0.0;
                    // the three one-way edge interpolants
                    v += (1 - eta) * (1 - zeta) * comp(ex[0], c) + eta * (1 - zeta) * comp(ex[1], c) +
                         (1 - eta) * zeta * comp(ex[2], c) + eta * zeta * comp(ex[3], c);
                    v += (1 - xi) * (1 - zeta) * comp(ee[0], c) + xi * (1 - zeta) * comp(ee[1], c) +
                         (1 - xi) * zeta * comp(ee[2], c) + xi * zeta * comp(ee[3], c);
                    v += (1 - xi) * (1 - eta) * comp(ez[0], c) + xi * (1 - eta) * comp(ez[1], c) +
                         (1 - xi) * eta * comp(ez[2], c) + xi * eta * comp(ez[3], c);
                    // minus the bilinear vertex surfaces of each pair of axes,
                    // blended across the third
                    const double f_k0 = (1 - xi) * (1 - eta) * comp(V[0], c) + xi * (1 - eta) * comp(V[1], c) +
                                        (1 - xi) * eta * comp(V[3], c) + xi * eta * comp(V[2], c);
                    const double f_k1 = (1 - xi) * (1 - eta) * comp(V[4], c) + xi * (1 - eta) * comp(V[5], c) +
                                        (1 - xi) * eta * comp(V[7], c) + xi * eta * comp(V[6], c);
                    v -= (1 - zeta) * f_k0 + zeta * f_k1;
                    const double f_i0 = (1 - eta) * (1 - zeta) * comp(V[0], c) + eta * (1 - zeta) * comp(V[3], c) +
                                        (1 - eta) * zeta * comp(V[4], c) + eta * zeta * comp(V[7], c);
                    const double f_i1 = (1 - eta) * (1 - zeta) * comp(V[1], c) + eta * (1 - zeta) * comp(V[2], c) +
                                        (1 - eta) * zeta * comp(V[5], c) + eta * zeta * comp(V[6], c);
                    v -= (1 - xi) * f_i0 + xi * f_i1;
                    const double f_j0 = (1 - xi) * (1 - zeta) * comp(V[0], c) + xi * (1 - zeta) * comp(V[1], c) +
                                        (1 - xi) * zeta * comp(V[4], c) + xi * zeta * comp(V[5], c);
                    const double f_j1 = (1 - xi) * (1 - zeta) * comp(V[3], c) + xi * (1 - zeta) * comp(V[2], c) +
                                        (1 - xi) * zeta * comp(V[7], c) + xi * zeta * comp(V[6], c);
                    v -= (1 - eta) * f_j0 + eta * f_j1;
                    // plus the trilinear vertex term
                    v += (1 - xi) * (1 - eta) * (1 - zeta) * comp(V[0], c) + xi * (1 - eta) * (1 - zeta) * comp(V[1], c) +
                         (1 - xi) * eta * (1 - zeta) * comp(V[3], c) + xi * eta * (1 - zeta) * comp(V[2], c) +
                         (1 - xi) * (1 - eta) * zeta * comp(V[4], c) + xi * (1 - eta) * zeta * comp(V[5], c) +
                         (1 - xi) * eta * zeta * comp(V[7], c) + xi * eta * zeta * comp(V[6], c);
                    p[c] = v;
                }
                x[idx] = p[0];
                y[idx] = p[1];
                z[idx] = p[2];
            }
        }
    }
}

FieldGeometry field_geometry(const MeshGeneration& m, int ng, const bool active[3]) {
    FieldGeometry F;
    F.ng = ng;
    int n[3];
    for (int d = 0; d < 3; ++d) {
        n[d] = m.cells[d] + 1;
        F.ext[d] = n[d] + 2 * ng;
    }
    const int MX = F.ext[0], MY = F.ext[1], MZ = F.ext[2];
    const size_t total = (size_t)MX * MY * MZ;
    F.x.assign(total, 0.0);
    F.y.assign(total, 0.0);
    F.z.assign(total, 0.0);
    {
        std::vector<double> bx, by, bz;
        block_points(m, bx, by, bz);
        size_t c = 0;
        for (int k = 0; k < n[2]; ++k)
            for (int j = 0; j < n[1]; ++j)
                for (int i = 0; i < n[0]; ++i, ++c) {
                    const long long t = F.at(i + ng, j + ng, k + ng);
                    F.x[t] = bx[c];
                    F.y[t] = by[c];
                    F.z[t] = bz[c];
                }
    }
    std::vector<double>* X[3] = {&F.x, &F.y, &F.z};
    // ghost coordinates: P = 2 P_near - P_far, axis by axis over the whole
    // extent of the other two axes (generateGhostCells, SF_mesh.cpp:491-533)
    auto extrapolate = [&](long long t, long long near, long long far) {
        for (int c = 0; c < 3; ++c) (*X[c])[t] = 2.0 * (*X[c])[near] - (*X[c])[far];
    };
    for (int k = 0; k < MZ; ++k)
        for (int j = 0; j < MY; ++j) {
            for (int i = ng - 1; i >= 0; --i) extrapolate(F.at(i, j, k), F.at(i + 1, j, k), F.at(i + 2, j, k));
            for (int i = MX - ng; i < MX; ++i) extrapolate(F.at(i, j, k), F.at(i - 1, j, k), F.at(i - 2, j, k));
        }
    for (int k = 0; k < MZ; ++k)
        for (int i = 0; i < MX; ++i) {
            for (int j = ng - 1; j >= 0; --j) extrapolate(F.at(i, j, k), F.at(i, j + 1, k), F.at(i, j + 2, k));
            for (int j = MY - ng; j < MY; ++j) extrapolate(F.at(i, j, k), F.at(i, j - 1, k), F.at(i, j - 2, k));
        }
    for (int j = 0; j < MY; ++j)
        for (int i = 0; i < MX; ++i) {
            for (int k = ng - 1; k >= 0; --k) extrapolate(F.at(i, j, k), F.at(i, j, k + 1), F.at(i, j, k + 2));
            for (int k = MZ - ng; k < MZ; ++k) extrapolate(F.at(i, j, k), F.at(i, j, k - 1), F.at(i, j, k - 2));
        }

    // metrics (computeMetrics, SF_mesh.cpp:219-345)
    const long long stride[3] = {1, MX, (long long)MX * MY};
    auto coord = [&](int c, long long t) { return (*X[c])[t]; };
    // central difference of coordinate c along axis a at point t
    auto dcoord = [&](int c, int a, long long t) {
        return 0.5 * (coord(c, t + stride[a]) - coord(c, t - stride[a]));
    };
    // central difference along `outer` of x_p * (d x_q / d inner)
    auto dproduct = [&](int p, int q, int inner, int outer, long long t) {
        const long long up = t + stride[outer], dn = t - stride[outer];
        const double hi = coord(p, up) * dcoord(q, inner, up);
        const double lo = coord(p, dn) * dcoord(q, inner, dn);
        return 0.5 * (hi - lo);
    };
    // symmetric conservative (Thomas-Lombard / SCMM) cofactor: the mean of
    // the two curl forms, with the cyclic successors of the axis and of the
    // component
    static const int after1[3] = {1, 2, 0}, after2[3] = {2, 0, 1};
    auto cofactor = [&](int axis, int c, long long t) {
        const int a = after1[axis], b = after2[axis];
        const int p = after1[c], q = after2[c];
        const double curl1 = dproduct(p, q, b, a, t) - dproduct(p, q, a, b, t);
        const double curl2 = dproduct(q, p, a, b, t) - dproduct(q, p, b, a, t);
        return 0.5 * (curl1 + curl2);
    };
    F.metrics.assign(total * 10, 0.0);
    for (int k = 1; k < MZ - 1; ++k)
        for (int j = 1; j < MY - 1; ++j)
            for (int i = 1; i < MX - 1; ++i) {
                const long long t = F.at(i, j, k);
                double r[3][3], cf[3][3];  // [axis][component]
                for (int a = 0; a < 3; ++a)
                    for (int c = 0; c < 3; ++c) r[a][c] = dcoord(c, a, t);
                for (int a = 0; a < 3; ++a)
                    for (int c = 0; c < 3; ++c) cf[a][c] = cofactor(a, c, t);
                auto rowdot = [&](int a) { return r[a][0] * cf[a][0] + r[a][1] * cf[a][1] + r[a][2] * cf[a][2]; };
                const double J = (rowdot(0) + rowdot(1) + rowdot(2)) / 3.0;
                if (!std::isfinite(J) || std::fabs(J) < 1e-18)
                    throw std::runtime_error("mesh: degenerate Jacobian at Field point (" + std::to_string(i) + "," +
                                             std::to_string(j) + "," + std::to_string(k) + ")");
                double* M = &F.metrics[t * 10];
                M[0] = 1.0 / J;
                for (int a = 0; a < 3; ++a)
                    for (int c = 0; c < 3; ++c) M[1 + 3 * a + c] = cf[a][c] * M[0];
            }
    // outermost layer: copies of the inner neighbour, i then j then k
    // (applyBoundaryMetrics, SF_mesh.cpp:439-474)
    auto copy = [&](long long dst, long long src) {
        std::copy(&F.metrics[src * 10], &F.metrics[src * 10] + 10, &F.metrics[dst * 10]);
    };
    for (int k = 0; k < MZ; ++k)
        for (int j = 0; j < MY; ++j) {
            copy(F.at(0, j, k), F.at(1, j, k));
            copy(F.at(MX - 1, j, k), F.at(MX - 2, j, k));
        }
    for (int k = 0; k < MZ; ++k)
        for (int i = 0; i < MX; ++i) {
            copy(F.at(i, 0, k), F.at(i, 1, k));
            copy(F.at(i, MY - 1, k), F.at(i, MY - 2, k));
        }
    for (int j = 0; j < MY; ++j)
        for (int i = 0; i < MX; ++i) {
            copy(F.at(i, j, 0), F.at(i, j, 1));
            copy(F.at(i, j, MZ - 1), F.at(i, j, MZ - 2));
        }

    // metric identity audit over the nodes and the active axes
    // (auditMetricIdentity, SF_mesh.cpp:348-437); face cofactors as the
    // canonical face builds them (SF_canonicalFace.h:56-118)
    auto face = [&](int axis, int c, long long t) {
        const double* A = &F.metrics[t * 10];
        const double* B = &F.metrics[(t + stride[axis]) * 10];
        if (!std::isfinite(A[0]) || !std::isfinite(B[0]) || std::fabs(A[0]) < 1e-30 || std::fabs(B[0]) < 1e-30)
            throw std::runtime_error("mesh: invalid inverse Jacobian at a face");
        return 0.5 * (A[1 + 3 * axis + c] / A[0] + B[1 + 3 * axis + c] / B[0]);
    };
    double worst = 0.0, cmax = 0.0;
    for (int k = ng; k < n[2] + ng; ++k)
        for (int j = ng; j < n[1] + ng; ++j)
            for (int i = ng; i < n[0] + ng; ++i) {
                const long long t = F.at(i, j, k);
                for (int c = 0; c < 3; ++c) {
                    double div = 0.0;
                    for (int a = 0; a < 3; ++a) {
                        if (!active[a]) continue;
                        const double fp = face(a, c, t), fm = face(a, c, t - stride[a]);
                        cmax = std::max({cmax, std::fabs(fp), std::fabs(fm)});
                        div += fp - fm;
                    }
                    if (!std::isfinite(div))
                        throw std::runtime_error("mesh: non-finite metric identity residual");
                    worst = std::max(worst, std::fabs(div));
                }
            }
    F.identity_residual = worst;
    F.identity_tolerance = 65536.0 * DBL_EPSILON * std::max(cmax, DBL_MIN);
    return F;
}

}  // namespace sfh
