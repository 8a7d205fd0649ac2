// sfh_vts.cpp -- ASCII .vts writer (see sfh_vts.hpp).
#include "sfh_vts.hpp"

#include <fstream>
#include <iomanip>

namespace sfh {

bool write_vts(const std::string& path, const VtsGeometry& geo, const std::vector<double>& q, double gamma,
               double time) {
    std::ofstream out(path);
    if (!out) return false;
    out << std::setprecision(17);
    const int nx = geo.nodes[0], ny = geo.nodes[1], nz = geo.nodes[2];
    const std::string ext =
        "0 " + std::to_string(nx - 1) + " 0 " + std::to_string(ny - 1) + " 0 " + std::to_string(nz - 1);
    out << "<?xml version=\"1.0\"?>\n"
        << "<VTKFile type=\"StructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\">\n"
        << "  <StructuredGrid WholeExtent=\"" << ext << "\">\n"
        << "    <FieldData>\n"
        << "      <DataArray type=\"Float64\" Name=\"TIME\" NumberOfTuples=\"1\" format=\"ascii\">" << time
        << "</DataArray>\n"
        << "    </FieldData>\n"
        << "    <Piece Extent=\"" << ext << "\">\n"
        << "      <Points>\n"
        << "        <DataArray type=\"Float64\" NumberOfComponents=\"3\" format=\"ascii\">\n";
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j) {
            for (int i = 0; i < nx; ++i) {
                if (geo.points) {
                    const double* p = &(*geo.points)[((size_t(k) * ny + j) * nx + i) * 3];
                    out << p[0] << ' ' << p[1] << ' ' << p[2] << ' ';
                } else {
                    out << geo.origin[0] + i * geo.h[0] << ' ' << geo.origin[1] + j * geo.h[1] << ' '
                        << geo.origin[2] + k * geo.h[2] << ' ';
                }
            }
            out << '\n';
        }
    out << "        </DataArray>\n      </Points>\n      <PointData Scalars=\"rho\" Vectors=\"U\">\n";
    const size_t nodes = size_t(nx) * ny * nz;
    auto array = [&](const char* name, int comps, auto&& value) {
        out << "        <DataArray type=\"Float64\" Name=\"" << name << "\" NumberOfComponents=\"" << comps
            << "\" format=\"ascii\">\n";
        for (size_t n = 0; n < nodes; ++n) {
            const double* s = &q[n * 5];
            for (int c = 0; c < comps; ++c) out << value(s, c) << ' ';
            if ((n + 1) % size_t(nx) == 0) out << '\n';
        }
        out << "        </DataArray>\n";
    };
    array("rho", 1, [](const double* s, int) { return s[0]; });
    array("U", 3, [](const double* s, int c) { return s[1 + c] / s[0]; });
    array("p", 1, [gamma](const double* s, int) {
        return (gamma - 1.0) * (s[4] - 0.5 * (s[1] * s[1] + s[2] * s[2] + s[3] * s[3]) / s[0]);
    });
    array("E", 1, [](const double* s, int) { return s[4]; });
    out << "      </PointData>\n    </Piece>\n  </StructuredGrid>\n</VTKFile>\n";
    return bool(out);
}

}  // namespace sfh
