// Test program: a reference-style main loop written against the drop-in
// headers (Particle, Step, computeAdaptiveDt, LoadParticlesFromFile), as a
// user of the reference would write it.  Prints the final state at full
// precision, one body per line.
//   dropin_step <ic.txt> <dt> <nsteps> <adaptive 0|1>
#include <cstdio>
#include <cstdlib>

#include "dt/adaptive.h"
#include "gravity/step.h"
#include "io/load_particle.hpp"

int main(int argc, char** argv) {
    if (argc != 5) return 1;
    Particle ps = LoadParticlesFromFile(argv[1]);
    const real dt = std::atof(argv[2]);
    const int nsteps = std::atoi(argv[3]);
    const bool adaptive = std::atoi(argv[4]) != 0;
    for (int s = 0; s < nsteps; ++s) {
        const real h = adaptive ? computeAdaptiveDt(ps, dt) : dt;
        Step(ps, h);
    }
    for (size_t i = 0; i < ps.size(); ++i)
        std::printf("%.17g %.17g %.17g %.17g %.17g %.17g\n", ps.x[i], ps.y[i], ps.z[i], ps.vx[i], ps.vy[i], ps.vz[i]);
    return 0;
}
