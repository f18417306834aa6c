// Legacy ASCII VTK snapshot in the reference's layout (src/io/vtk_save.h:21-75):
// POLYDATA points, one vertex per body, point data `type`, `velocity`, `mass`.
// Numbers use the default iostream formatting, as the reference writes them.
// The data type name follows `real` (double with NEXT_FP64, float with
// NEXT_FP32), which is the reference's rule wherever the reference compiles.
#pragma once
#include <fstream>
#include <string>
#include <type_traits>

#include "../struct/particle.h"

inline void SaveVTK(const Particle& p, const std::string& filename) {
    std::ofstream out(filename);
    if (!out) return;
    const size_t n = p.size();
    const char* t = std::is_same<real, double>::value ? "double" : "float";
    out << "# vtk DataFile Version 3.0\nNEXT snapshot\nASCII\nDATASET POLYDATA\n";
    out << "POINTS " << n << " " << t << "\n";
    for (size_t i = 0; i < n; ++i) out << p.x[i] << " " << p.y[i] << " " << p.z[i] << "\n";
    out << "VERTICES " << n << " " << n * 2 << "\n";
    for (size_t i = 0; i < n; ++i) out << "1 " << i << "\n";
    out << "POINT_DATA " << n << "\n";
    out << "SCALARS type int 1\nLOOKUP_TABLE default\n";
    for (size_t i = 0; i < n; ++i) out << p.type[i] << "\n";
    out << "VECTORS velocity " << t << "\n";
    for (size_t i = 0; i < n; ++i) out << p.vx[i] << " " << p.vy[i] << " " << p.vz[i] << "\n";
    out << "SCALARS mass " << t << " 1\nLOOKUP_TABLE default\n";
    for (size_t i = 0; i < n; ++i) out << p.m[i] << "\n";
}
