// ASCII VTU (XML UnstructuredGrid) snapshot in the reference's layout
// (src/io/vtu_save.h:22-78): one VTK_VERTEX cell per body, point data
// `type`, `velocity`, `mass`.
#pragma once
#include <fstream>
#include <string>

#include "../struct/particle.h"

inline void SaveVTU(const Particle& p, const std::string& filename) {
    std::ofstream out(filename);
    if (!out) return;
    const size_t n = p.size();
    out << "<?xml version=\"1.0\"?>\n"
        << "<VTKFile type=\"UnstructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\">\n"
        << "  <UnstructuredGrid>\n"
        << "    <Piece NumberOfPoints=\"" << n << "\" NumberOfCells=\"" << n << "\">\n";
    out << "      <Points>\n        <DataArray type=\"Float32\" NumberOfComponents=\"3\" format=\"ascii\">\n          ";
    for (size_t i = 0; i < n; ++i) out << p.x[i] << " " << p.y[i] << " " << p.z[i] << " ";
    out << "\n        </DataArray>\n      </Points>\n";
    out << "      <Cells>\n        <DataArray type=\"Int32\" Name=\"connectivity\" format=\"ascii\">\n          ";
    for (size_t i = 0; i < n; ++i) out << i << " ";
    out << "\n        </DataArray>\n        <DataArray type=\"Int32\" Name=\"offsets\" format=\"ascii\">\n          ";
    for (size_t i = 1; i <= n; ++i) out << i << " ";
    out << "\n        </DataArray>\n        <DataArray type=\"UInt8\" Name=\"types\" format=\"ascii\">\n          ";
    for (size_t i = 0; i < n; ++i) out << "1 ";
    out << "\n        </DataArray>\n      </Cells>\n      <PointData>\n";
    out << "        <DataArray type=\"Int32\" Name=\"type\" format=\"ascii\">\n          ";
    for (size_t i = 0; i < n; ++i) out << p.type[i] << " ";
    out << "\n        </DataArray>\n";
    out << "        <DataArray type=\"Float32\" Name=\"velocity\" NumberOfComponents=\"3\" format=\"ascii\">\n          ";
    for (size_t i = 0; i < n; ++i) out << p.vx[i] << " " << p.vy[i] << " " << p.vz[i] << " ";
    out << "\n        </DataArray>\n";
    out << "        <DataArray type=\"Float32\" Name=\"mass\" format=\"ascii\">\n          ";
    for (size_t i = 0; i < n; ++i) out << p.m[i] << " ";
    out << "\n        </DataArray>\n      </PointData>\n    </Piece>\n  </UnstructuredGrid>\n</VTKFile>\n";
}
