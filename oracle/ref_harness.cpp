// Test infrastructure only: a C-ABI harness around NEXT's own gravity code.
//
// This file contains no copy of the reference.  It is compiled with
//   -I<reference>/src -I<reference>/include -DNEXT_FP64
// so that the #includes below pull in the unmodified reference headers
// (src/gravity/step.h, src/gravity/octree.h, src/dt/softening.h,
//  src/dt/adaptive.h, src/struct/particle.h, include/floatdef.h, and the
//  snapshot writers src/io/vtk_save.h, src/io/vtu_save.h).
// The resulting oracle/_ref/libnextref.so is used by the tests as the
// ground truth for reference-semantics parity, by tests/golden/make_golden.py
// to produce the committed fixtures, and by bench.py as the timed CPU
// baseline (the reference's own OpenMP Step()).  Nothing in the product
// links or loads it.
#include "gravity/step.h"
#include "dt/adaptive.h"
#include "io/vtk_save.h"
#include "io/vtu_save.h"

#include <cstdint>
#include <functional>
#include <omp.h>

namespace {

Particle make_particles(int64_t n, const double* x, const double* y, const double* z,
                        const double* vx, const double* vy, const double* vz,
                        const double* m, const int* type) {
    Particle p;
    p.resize(static_cast<size_t>(n));
    for (int64_t i = 0; i < n; ++i) {
        p.x[i] = x[i]; p.y[i] = y[i]; p.z[i] = z[i];
        p.vx[i] = vx ? vx[i] : 0.0; p.vy[i] = vy ? vy[i] : 0.0; p.vz[i] = vz ? vz[i] : 0.0;
        p.m[i] = m[i];
        p.type[i] = type ? type[i] : 0;
    }
    return p;
}

// The reference builds its tree inside a lambda local to Step()
// (src/gravity/step.h:67-109), which cannot be called from outside.  The
// harness therefore repeats that lambda's two bookkeeping lines -- the
// bounding box and the root cube -- and then calls the reference's own
// Octree::insert and Octree::computeMass, exactly in the lambda's order.
std::unique_ptr<Octree> build_reference_tree(const Particle& ps) {
    const int N = static_cast<int>(ps.size());
    double lo[3] = {1e30, 1e30, 1e30}, hi[3] = {-1e30, -1e30, -1e30};
    for (int i = 0; i < N; ++i) {
        lo[0] = std::min(lo[0], ps.x[i]); hi[0] = std::max(hi[0], ps.x[i]);
        lo[1] = std::min(lo[1], ps.y[i]); hi[1] = std::max(hi[1], ps.y[i]);
        lo[2] = std::min(lo[2], ps.z[i]); hi[2] = std::max(hi[2], ps.z[i]);
    }
    const double cx = (lo[0] + hi[0]) * 0.5;
    const double cy = (lo[1] + hi[1]) * 0.5;
    const double cz = (lo[2] + hi[2]) * 0.5;
    double half = std::max({hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]}) * 0.5;
    if (half <= 0.0) half = 1.0;
    auto root = std::make_unique<Octree>(cx, cy, cz, half);
    for (int i = 0; i < N; ++i) root->insert(i, ps);
    root->computeMass(ps);
    return root;
}

}  // namespace

extern "C" {

void ref_set_threads(int threads) {
    if (threads > 0) omp_set_num_threads(threads);
}

int ref_max_threads(void) { return omp_get_max_threads(); }

// Per-particle accelerations exactly as one kick of the reference computes them
// (tree of src/gravity/step.h:67-109, bhAccel of src/gravity/octree.h:133 with
// theta = 0.5 as hard-coded at step.h:32).
int ref_accel(int64_t n, const double* x, const double* y, const double* z,
              const double* m, const int* type, double theta,
              double* ax, double* ay, double* az) {
    if (n <= 0) return 0;
    Particle ps = make_particles(n, x, y, z, nullptr, nullptr, nullptr, m, type);
    auto root = build_reference_tree(ps);
    #pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < n; ++i) {
        double a0 = 0, a1 = 0, a2 = 0;
        bhAccel(root.get(), static_cast<int>(i), ps, theta, a0, a1, a2);
        ax[i] = a0; ay[i] = a1; az[i] = a2;
    }
    return 0;
}

// The same accelerations for the k bodies listed in idx only (one tree, k
// walks): the reference's as-shipped force on a sample.
int ref_accel_sample(int64_t n, const double* x, const double* y, const double* z,
                     const double* m, const int* type, double theta, int64_t k, const int64_t* idx,
                     double* ax, double* ay, double* az) {
    if (n <= 0) return 0;
    Particle ps = make_particles(n, x, y, z, nullptr, nullptr, nullptr, m, type);
    auto root = build_reference_tree(ps);
    #pragma omp parallel for schedule(dynamic, 16)
    for (int64_t t = 0; t < k; ++t) {
        double a0 = 0, a1 = 0, a2 = 0;
        bhAccel(root.get(), static_cast<int>(idx[t]), ps, theta, a0, a1, a2);
        ax[t] = a0; ay[t] = a1; az[t] = a2;
    }
    return 0;
}

// nsteps calls of the reference's Step() (src/gravity/step.h:25), in place.
int ref_step(int64_t n, double* x, double* y, double* z,
             double* vx, double* vy, double* vz,
             const double* m, const int* type, double dt, int nsteps) {
    Particle ps = make_particles(n, x, y, z, vx, vy, vz, m, type);
    for (int s = 0; s < nsteps; ++s) Step(ps, dt);
    for (int64_t i = 0; i < n; ++i) {
        x[i] = ps.x[i]; y[i] = ps.y[i]; z[i] = ps.z[i];
        vx[i] = ps.vx[i]; vy[i] = ps.vy[i]; vz[i] = ps.vz[i];
    }
    return 0;
}

// The reference's adaptive time step (src/dt/adaptive.h:23).
double ref_adaptive_dt(int64_t n, const double* vx, const double* vy, const double* vz,
                       double base_dt) {
    Particle ps;
    ps.resize(static_cast<size_t>(n));
    for (int64_t i = 0; i < n; ++i) { ps.vx[i] = vx[i]; ps.vy[i] = vy[i]; ps.vz[i] = vz[i]; }
    return computeAdaptiveDt(ps, base_dt);
}

// The reference's softening law (src/dt/softening.h:21).
double ref_next_softening(double size, double mass, double dist) {
    return nextSoftening(size, mass, dist);
}

// Depth-first export of the reference octree (children visited 0..7, the
// order bhAccel uses).  One row of 16 doubles per node:
//   level, m, comx, comy, comz, half_width, Qxx, Qyy, Qzz, Qxy, Qxz, Qyz,
//   leaf, body_index, centre_x, octant_path_low_bits
// Returns the node count (rows written up to cap).
int64_t ref_tree_export(int64_t n, const double* x, const double* y, const double* z,
                        const double* m, double* rows, int64_t cap) {
    if (n <= 0) return 0;
    Particle ps = make_particles(n, x, y, z, nullptr, nullptr, nullptr, m, nullptr);
    auto root = build_reference_tree(ps);
    int64_t count = 0;
    std::function<void(const Octree*, int)> visit = [&](const Octree* nd, int level) {
        if (count < cap) {
            double* r = rows + 16 * count;
            r[0] = level; r[1] = nd->m; r[2] = nd->cx; r[3] = nd->cy; r[4] = nd->cz;
            r[5] = nd->size; r[6] = nd->Qxx; r[7] = nd->Qyy; r[8] = nd->Qzz;
            r[9] = nd->Qxy; r[10] = nd->Qxz; r[11] = nd->Qyz;
            r[12] = nd->leaf ? 1.0 : 0.0; r[13] = nd->bodyIdx; r[14] = nd->x; r[15] = 0.0;
        }
        ++count;
        for (int c = 0; c < 8; ++c)
            if (nd->child[c]) visit(nd->child[c].get(), level + 1);
    };
    visit(root.get(), 0);
    return count;
}

// For every particle, the octant digits of the path from the root to its leaf
// in the reference tree, packed 3 bits per level from the top of a 64-bit word
// (level 1 in bits 62..60), and the leaf depth.  The walk down uses the
// reference's own Octree::getOctant and child pointers.
int ref_leaf_paths(int64_t n, const double* x, const double* y, const double* z,
                   const double* m, uint64_t* paths, int* depth) {
    if (n <= 0) return 0;
    Particle ps = make_particles(n, x, y, z, nullptr, nullptr, nullptr, m, nullptr);
    auto root = build_reference_tree(ps);
    for (int64_t i = 0; i < n; ++i) {
        const Octree* nd = root.get();
        uint64_t key = 0;
        int lvl = 0;
        while (!nd->leaf) {
            int oct = nd->getOctant(ps.x[i], ps.y[i], ps.z[i]);
            ++lvl;
            if (lvl <= 21) key |= static_cast<uint64_t>(oct) << (63 - 3 * lvl);
            nd = nd->child[oct].get();
            if (!nd) return -1;
        }
        if (nd->bodyIdx != static_cast<int>(i)) return -2;
        paths[i] = key;
        depth[i] = lvl;
    }
    return 0;
}

// A snapshot written by the reference's own writers: SaveVTK
// (src/io/vtk_save.h:21-75) or SaveVTU (src/io/vtu_save.h:22-78).
int ref_save_snapshot(int64_t n, const double* x, const double* y, const double* z,
                      const double* vx, const double* vy, const double* vz,
                      const double* m, const int* type, int vtu, const char* path) {
    Particle p = make_particles(n, x, y, z, vx, vy, vz, m, type);
    if (vtu) SaveVTU(p, path);
    else SaveVTK(p, path);
    return 0;
}

}  // extern "C"
