// Drop-in computeAdaptiveDt() (src/dt/adaptive.h:23-52): the largest body
// speed is found by a device reduction, then dt = base/(1+v) clamped to
// [base/100, base], with v capped at 1e4 and base returned for v < 1e-8.
#pragma once
#include "../floatdef.h"
#include "../gravity/engine.h"
#include "../struct/particle.h"

inline real computeAdaptiveDt(const Particle& p, real base_dt) {
    if (p.size() == 0) return base_dt;
    next_gpu::Engine& e = next_gpu::engine();
    e.upload(p);
    return static_cast<real>(e.adaptive_dt(static_cast<double>(base_dt)));
}
