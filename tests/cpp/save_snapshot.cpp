// Test program: writes one snapshot with the drop-in writers SaveVTK / SaveVTU
// (next_b200/host/io), from a raw file of n bodies: 7 lanes of n doubles
// (x y z vx vy vz m) followed by n int32 types.
//   save_snapshot <bodies.bin> <n> <vtk|vtu> <out>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "io/vtk_save.h"
#include "io/vtu_save.h"

int main(int argc, char** argv) {
    if (argc != 5) return 1;
    const size_t n = std::strtoull(argv[2], nullptr, 10);
    std::FILE* f = std::fopen(argv[1], "rb");
    if (!f) return 2;
    std::vector<double> lanes(7 * n);
    std::vector<int> type(n);
    if (std::fread(lanes.data(), sizeof(double), 7 * n, f) != 7 * n) return 3;
    if (std::fread(type.data(), sizeof(int), n, f) != n) return 3;
    std::fclose(f);
    Particle p;
    p.resize(n);
    for (size_t i = 0; i < n; ++i) {
        p.x[i] = lanes[i]; p.y[i] = lanes[n + i]; p.z[i] = lanes[2 * n + i];
        p.vx[i] = lanes[3 * n + i]; p.vy[i] = lanes[4 * n + i]; p.vz[i] = lanes[5 * n + i];
        p.m[i] = lanes[6 * n + i];
        p.type[i] = type[i];
    }
    if (std::strcmp(argv[3], "vtu") == 0) SaveVTU(p, argv[4]);
    else SaveVTK(p, argv[4]);
    return 0;
}
