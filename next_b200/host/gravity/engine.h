// C++ owner of one libnext_b200 handle (include/next_gpu.h) for the drop-in
// Step()/computeAdaptiveDt() and the `next` driver.
//
// Configuration comes from next_gpu::configure() or, when that was not
// called, from the environment:
//   NEXT_PHYSICS   reference (default) | accurate
//   NEXT_PRECISION fp64 (default)      | mixed | fp64group   (the last two need accurate)
//   NEXT_THETA, NEXT_EPS, NEXT_LEAF_CAP, NEXT_DEVICE
// The default reproduces the reference's physics (theta 0.5 on half-widths,
// adaptive softening, its quadrupole) with FP64 arithmetic on the GPU.
#pragma once
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../../include/next_gpu.h"
#include "../struct/particle.h"

namespace next_gpu {

inline next_params params_from_env() {
    auto get = [](const char* k) -> const char* { return std::getenv(k); };
    const std::string phys = get("NEXT_PHYSICS") ? get("NEXT_PHYSICS") : "reference";
    const std::string prec = get("NEXT_PRECISION") ? get("NEXT_PRECISION") : "fp64";
    next_params p;
    next_params_default(&p, phys == "accurate" ? NEXT_PHYSICS_ACCURATE : NEXT_PHYSICS_REFERENCE,
                        prec == "mixed" ? NEXT_PRECISION_MIXED
                                        : prec == "fp64group" ? NEXT_PRECISION_FP64_GROUP : NEXT_PRECISION_FP64);
    if (get("NEXT_THETA")) p.theta = std::atof(get("NEXT_THETA"));
    if (get("NEXT_EPS")) p.eps = std::atof(get("NEXT_EPS"));
    if (get("NEXT_LEAF_CAP")) p.leaf_cap = std::atoi(get("NEXT_LEAF_CAP"));
    if (get("NEXT_DEVICE")) p.device = std::atoi(get("NEXT_DEVICE"));
    return p;
}

class Engine {
public:
    explicit Engine(const next_params& p) {
        const int rc = next_create(&p, &h_);
        if (rc != NEXT_OK) throw std::runtime_error(std::string("next_create: ") + next_status_string(rc));
    }
    ~Engine() { next_destroy(h_); }
    Engine(const Engine&) = delete;
    Engine& operator=(const Engine&) = delete;

    next_handle* handle() const { return h_; }

    void check(int rc, const char* what) const {
        if (rc != NEXT_OK)
            throw std::runtime_error(std::string(what) + ": " + next_status_string(rc) + ": " + next_last_error(h_));
    }

    // Host -> device.  Unchanged positions and masses keep the tree order and
    // the forces cached by the previous step.
    void upload(const Particle& ps) {
        const int64_t n = static_cast<int64_t>(ps.size());
#if defined(NEXT_FP32)
        std::vector<double> lanes[7];
        const std::vector<real>* src[7] = {&ps.x, &ps.y, &ps.z, &ps.vx, &ps.vy, &ps.vz, &ps.m};
        for (int c = 0; c < 7; ++c) lanes[c].assign(src[c]->begin(), src[c]->end());
        check(next_upload(h_, n, lanes[0].data(), lanes[1].data(), lanes[2].data(), lanes[3].data(),
                          lanes[4].data(), lanes[5].data(), lanes[6].data(), ps.type.data()), "upload");
#else
        check(next_upload(h_, n, ps.x.data(), ps.y.data(), ps.z.data(), ps.vx.data(), ps.vy.data(), ps.vz.data(),
                          ps.m.data(), ps.type.data()), "upload");
#endif
    }

    // Device -> host (positions and velocities, the lanes a step changes).
    void download(Particle& ps) {
#if defined(NEXT_FP32)
        const size_t n = ps.size();
        std::vector<double> lanes[6];
        for (auto& l : lanes) l.resize(n);
        check(next_download(h_, lanes[0].data(), lanes[1].data(), lanes[2].data(), lanes[3].data(),
                            lanes[4].data(), lanes[5].data()), "download");
        std::vector<real>* dst[6] = {&ps.x, &ps.y, &ps.z, &ps.vx, &ps.vy, &ps.vz};
        for (int c = 0; c < 6; ++c) dst[c]->assign(lanes[c].begin(), lanes[c].end());
#else
        check(next_download(h_, ps.x.data(), ps.y.data(), ps.z.data(), ps.vx.data(), ps.vy.data(), ps.vz.data()),
              "download");
#endif
    }

    void step(double dt) { check(next_step(h_, dt), "step"); }

    // Upload, one step and the copy back in one call; the positions travel
    // back while the force phase runs.
    void step_host(Particle& ps, double dt) {
        const int64_t n = static_cast<int64_t>(ps.size());
#if defined(NEXT_FP32)
        std::vector<double> lanes[7];
        std::vector<real>* src[7] = {&ps.x, &ps.y, &ps.z, &ps.vx, &ps.vy, &ps.vz, &ps.m};
        for (int c = 0; c < 7; ++c) lanes[c].assign(src[c]->begin(), src[c]->end());
        check(next_step_host(h_, dt, n, lanes[0].data(), lanes[1].data(), lanes[2].data(), lanes[3].data(),
                             lanes[4].data(), lanes[5].data(), lanes[6].data(), ps.type.data()), "step");
        for (int c = 0; c < 6; ++c) src[c]->assign(lanes[c].begin(), lanes[c].end());
#else
        check(next_step_host(h_, dt, n, ps.x.data(), ps.y.data(), ps.z.data(), ps.vx.data(), ps.vy.data(),
                             ps.vz.data(), ps.m.data(), ps.type.data()), "step");
#endif
    }

    double adaptive_dt(double base) {
        double dt = base;
        check(next_adaptive_dt(h_, base, &dt), "adaptive dt");
        return dt;
    }

private:
    next_handle* h_ = nullptr;
};

// The process-wide engine behind Step()/computeAdaptiveDt().
inline Engine*& engine_slot() {
    static Engine* e = nullptr;
    return e;
}

inline void configure(const next_params& p) {
    delete engine_slot();
    engine_slot() = new Engine(p);
}

inline Engine& engine() {
    if (!engine_slot()) engine_slot() = new Engine(params_from_env());
    return *engine_slot();
}

}  // namespace next_gpu
