// sfh_vts.cpp -- ASCII .vts writer in the reference's result layout (see
// sfh_vts.hpp).
#include "sfh_vts.hpp"

#include <algorithm>
#include <fstream>
#include <iomanip>
#include <map>

namespace sfh {

namespace {

// Membership of written node (i, j, k) in a set of the structured generator
// (its boundary planes and named sets, src/infrastructure/mesh/createMesh/
// SF_meshGen.cpp:478-540); n: written nodes per axis.
bool in_set(const std::string& name, int i, int j, int k, const int n[3]) {
    const bool j_plane = n[1] > 1 && (j == 0 || j == n[1] - 1);
    const bool k_plane = n[2] > 1 && (k == 0 || k == n[2] - 1);
    if (name == "Left" || name == "inlet") return i == 0;
    if (name == "Right" || name == "outlet") return i == n[0] - 1;
    if (name == "sideWalls") return j_plane;
    if (name == "frontBack") return k_plane;
    if (name == "walls") return j_plane || k_plane;
    if (name == "all") return true;
    if (name == "leftHalf") return i < n[0] / 2;
    if (name == "rightHalf") return i >= n[0] / 2;
    return false;  // a name the generator has no set for marks nothing
}

void put_ids(std::ostream& out, const char* name, const std::vector<int>& ids, const int n[3]) {
    out << "        <DataArray type=\"Int32\" Name=\"" << name << "\" format=\"ascii\">\n";
    size_t t = 0;
    for (int k = 0; k < n[2]; ++k)
        for (int j = 0; j < n[1]; ++j) {
            for (int i = 0; i < n[0]; ++i) out << ids[t++] << " ";
            out << "\n";
        }
    out << "        </DataArray>\n";
}

}  // namespace

VtsLayout vts_layout(const CaseSpec& c, const GridSetup& g, const std::vector<double>& block_points) {
    VtsLayout L;
    for (int d = 0; d < 3; ++d) {
        L.nodes[d] = g.nodes[d];
        const bool periodic = g.grid.bc_lo[d] == SFG_BC_PERIODIC;
        L.out_nodes[d] = periodic ? g.nodes[d] : c.cells[d] + 1;
        L.origin[d] = c.lo[d];
        L.h[d] = (c.hi[d] - c.lo[d]) / c.cells[d];
    }
    const int* n = L.out_nodes;
    const size_t total = size_t(n[0]) * n[1] * n[2];
    if (!block_points.empty() && block_points.size() == total * 3) L.points = block_points;
    // boundary sets named by the conditions, numbered by first appearance
    // over rho, U, p (appendBoundaryZoneNames, SF_vtkUtils.h:43-51)
    std::vector<std::string> names;
    for (const char* var : {"rho", "U", "p"}) {
        auto it = c.bc_order.find(var);
        if (it == c.bc_order.end()) continue;
        for (const auto& s : it->second)
            if (std::find(names.begin(), names.end(), s) == names.end()) names.push_back(s);
    }
    for (auto& ids : L.bc_id) ids.assign(total, 0);
    const char* vars[3] = {"rho", "U", "p"};
    for (int v = 0; v < 3; ++v) {
        auto it = c.bc_order.find(vars[v]);
        if (it == c.bc_order.end()) continue;
        for (const auto& s : it->second) {  // later conditions win on shared nodes
            const int id = int(std::find(names.begin(), names.end(), s) - names.begin()) + 1;
            size_t t = 0;
            for (int k = 0; k < n[2]; ++k)
                for (int j = 0; j < n[1]; ++j)
                    for (int i = 0; i < n[0]; ++i, ++t)
                        if (in_set(s, i, j, k, n)) L.bc_id[1 + v][t] = id;
        }
    }
    for (size_t t = 0; t < total; ++t) {
        int id = L.bc_id[1][t];
        if (L.bc_id[2][t]) id = L.bc_id[2][t];
        if (L.bc_id[3][t]) id = L.bc_id[3][t];
        L.bc_id[0][t] = id;
    }
    for (size_t s = 0; s < names.size(); ++s) L.legend += ", " + std::to_string(s + 1) + "=" + names[s];
    // fluid arrays: the built-in names, taken over by the registry's
    // declarations (ModelLoader::configureOutput, SF_output.cpp:31-118)
    std::map<std::string, VtsQuantity> arrays{{"Density", VtsQuantity::Density},
                                              {"Velocity", VtsQuantity::Velocity},
                                              {"Pressure", VtsQuantity::Pressure}};
    const std::map<std::string, std::string> alias{{"rho", "Density"}, {"U", "Velocity"}, {"p", "Pressure"}};
    for (const auto& f : c.declared_fields) {
        if (!f.output) continue;
        auto it = arrays.find(f.name);
        if (it == arrays.end()) {
            auto a = alias.find(f.name);
            if (a != alias.end()) it = arrays.find(a->second);
        }
        if (it == arrays.end()) it = arrays.find(f.output_name);
        if (it == arrays.end()) continue;  // a field this path has no values for
        const VtsQuantity q = it->second;
        arrays.erase(it);
        arrays[f.output_name] = q;
    }
    for (const auto& kv : arrays) L.arrays.push_back({kv.first, kv.second});
    return L;
}

bool write_vts(const std::string& path, const VtsLayout& geo, const std::vector<double>& q, double gamma) {
    std::ofstream out(path);
    if (!out) return false;
    out << std::setprecision(17);
    const int* n = geo.out_nodes;
    const std::string ext =
        "0 " + std::to_string(n[0] - 1) + " 0 " + std::to_string(n[1] - 1) + " 0 " + std::to_string(n[2] - 1);
    out << "<?xml version=\"1.0\"?>\n"
        << "<VTKFile type=\"StructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\">\n"
        << "  <StructuredGrid WholeExtent=\"" << ext << "\">\n"
        << "    <Piece Extent=\"" << ext << "\">\n"
        << "      <Points>\n"
        << "        <DataArray type=\"Float64\" NumberOfComponents=\"3\" format=\"ascii\">\n";
    size_t t = 0;
    for (int k = 0; k < n[2]; ++k)
        for (int j = 0; j < n[1]; ++j) {
            for (int i = 0; i < n[0]; ++i, ++t) {
                if (!geo.points.empty()) {
                    const double* p = &geo.points[t * 3];
                    out << p[0] << " " << p[1] << " " << p[2] << " ";
                } else {
                    out << geo.origin[0] + i * geo.h[0] << " " << geo.origin[1] + j * geo.h[1] << " "
                        << geo.origin[2] + k * geo.h[2] << " ";
                }
            }
            out << "\n";
        }
    out << "        </DataArray>\n      </Points>\n      <PointData>\n";
    put_ids(out, "BC_ID", geo.bc_id[0], n);
    put_ids(out, "BC_ID_rho", geo.bc_id[1], n);
    put_ids(out, "BC_ID_U", geo.bc_id[2], n);
    put_ids(out, "BC_ID_p", geo.bc_id[3], n);
    out << "        <!-- BC_ID legend: 0=interior/internal-shared/unconfigured" << geo.legend
        << "; variable BC_ID arrays use the same legend and follow per-variable boundaryField order on overlaps"
           " -->\n";
    // the provider's node of a written node: an unsolved axis has one
    auto state = [&](int i, int j, int k) {
        const int ii = geo.nodes[0] > 1 ? i : 0, jj = geo.nodes[1] > 1 ? j : 0, kk = geo.nodes[2] > 1 ? k : 0;
        return &q[((size_t(kk) * geo.nodes[1] + jj) * geo.nodes[0] + ii) * 5];
    };
    for (const auto& a : geo.arrays) {
        const int comps = a.what == VtsQuantity::Velocity ? 3 : 1;
        out << "        <DataArray type=\"Float64\" Name=\"" << a.name << "\" NumberOfComponents=\"" << comps
            << "\" format=\"ascii\">\n";
        for (int k = 0; k < n[2]; ++k)
            for (int j = 0; j < n[1]; ++j)
                for (int i = 0; i < n[0]; ++i) {
                    const double* s = state(i, j, k);
                    for (int c = 0; c < comps; ++c) {
                        double v;
                        if (a.what == VtsQuantity::Density) v = s[0];
                        else if (a.what == VtsQuantity::Velocity) v = s[1 + c] / s[0];
                        else v = (gamma - 1.0) * (s[4] - 0.5 * (s[1] * s[1] + s[2] * s[2] + s[3] * s[3]) / s[0]);
                        out << v << ' ';
                    }
                    out << '\n';
                }
        out << "        </DataArray>\n";
    }
    out << "      </PointData>\n    </Piece>\n  </StructuredGrid>\n</VTKFile>\n";
    return bool(out);
}

}  // namespace sfh
