// Drop-in Step(): one KDK leapfrog step of the whole system on the GPU, with
// the reference's signature and in-place semantics (src/gravity/step.h:25):
// kick dt/2 with forces at x_n, drift dt, kick dt/2 with forces at x_{n+1}.
// The bodies are uploaded (forces cached from the previous call are kept when
// the positions did not change), stepped on the device and copied back into
// ps, the positions while the force phase still runs.  Unlike the reference, failures throw std::runtime_error, and bodies at
// identical positions share a leaf instead of recursing without end.
#pragma once
#include "../floatdef.h"
#include "../struct/particle.h"
#include "engine.h"

inline void Step(ParticleSystem& ps, real dt) {
    if (ps.size() == 0) return;   // as src/gravity/step.h:26
    next_gpu::engine().step_host(ps, static_cast<double>(dt));
}
