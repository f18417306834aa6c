// Text initial conditions: whitespace-separated rows `x y z vx vy vz m type`,
// read until the first row that does not parse (the reference's text path,
// src/io/load_particle.hpp:100-116).  The reference first tries HDF5; this
// build has no libhdf5, so only the text format is read.
#pragma once
#include <fstream>
#include <string>

#include "../struct/particle.h"

inline Particle LoadParticlesFromFile(const std::string& filename) {
    Particle p;
    std::ifstream in(filename);
    real tx, ty, tz, tvx, tvy, tvz, tm;
    int tt;
    while (in >> tx >> ty >> tz >> tvx >> tvy >> tvz >> tm >> tt) p.addParticle(tx, ty, tz, tvx, tvy, tvz, tm, tt);
    return p;
}
