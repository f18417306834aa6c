// The reference's particle container, same lanes and members
// (src/struct/particle.h:22-57): x y z vx vy vz ax ay az m as `real` vectors
// and `type` as int.  Kept identical so code written against the reference
// compiles unchanged against this header.
#pragma once
#include <cstddef>
#include <vector>

#include "floatdef.h"

struct Particle {
    std::vector<real> x, y, z;
    std::vector<real> vx, vy, vz;
    std::vector<real> ax, ay, az;
    std::vector<real> m;
    std::vector<int> type;

    void resize(size_t n) {
        for (auto* v : {&x, &y, &z, &vx, &vy, &vz, &m}) v->resize(n, 0);
        for (auto* v : {&ax, &ay, &az}) v->assign(n, 0);
        type.resize(n, 0);
    }

    void addParticle(real px, real py, real pz, real pvx, real pvy, real pvz, real pm, int ptype) {
        x.push_back(px); y.push_back(py); z.push_back(pz);
        vx.push_back(pvx); vy.push_back(pvy); vz.push_back(pvz);
        ax.push_back(0); ay.push_back(0); az.push_back(0);
        m.push_back(pm);
        type.push_back(ptype);
    }

    size_t size() const { return x.size(); }

    void clear() {
        for (auto* v : {&x, &y, &z, &vx, &vy, &vz, &ax, &ay, &az, &m}) v->clear();
        type.clear();
    }
};

using ParticleSystem = Particle;
