// ORACLE -- test infrastructure only.
//
// A plain C++ (CPU, FP64) restatement of NEXT's gravity hot path, used by the
// tests and by bench.py's CPU-baseline leg as the checker for the CUDA
// library.  Nothing in the shipped library links, loads or calls this file.
// It is pinned against the reference itself: tests compare it with
// oracle/_ref/libnextref.so (the reference's own headers compiled by
// oracle/Makefile) and with the fixtures in tests/golden/.
//
// Two physics modes:
//   REF       -- the reference's semantics: one body per leaf, half-width
//                opening test size/dist < theta, adaptive softening, the
//                reference's quadrupole (child-COM-only moments with the
//                size^2/100 regulariser, and the sign used at
//                src/gravity/octree.h:170-172).
//   ACCURATE  -- the same tree walk with the physics corrected: Plummer
//                softening eps, full-width opening test with the COM offset
//                (d > l/theta + delta), traceless quadrupole with
//                parallel-axis terms and the correct sign, leaf buckets.
//
// Built with -ffp-contract=off so every + - * / is one IEEE operation in the
// order written, which is also the order the reference source gives.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>

namespace {

constexpr int kMaxLevel = 21;  // 3 bits per level in a 63-bit key

struct Cube { double cx, cy, cz, half; };

// Bounding box and root cube: src/gravity/step.h:69-100.
Cube root_cube(int64_t n, const double* x, const double* y, const double* z) {
    double lo[3] = {1e30, 1e30, 1e30}, hi[3] = {-1e30, -1e30, -1e30};
    for (int64_t i = 0; i < n; ++i) {
        lo[0] = std::min(lo[0], x[i]); hi[0] = std::max(hi[0], x[i]);
        lo[1] = std::min(lo[1], y[i]); hi[1] = std::max(hi[1], y[i]);
        lo[2] = std::min(lo[2], z[i]); hi[2] = std::max(hi[2], z[i]);
    }
    Cube c;
    c.cx = (lo[0] + hi[0]) * 0.5;
    c.cy = (lo[1] + hi[1]) * 0.5;
    c.cz = (lo[2] + hi[2]) * 0.5;
    c.half = std::max(std::max(hi[0] - lo[0], hi[1] - lo[1]), hi[2] - lo[2]) * 0.5;
    if (c.half <= 0.0) c.half = 1.0;
    return c;
}

// Octant key: the sequence of octants the reference's insertion would take.
// At every level the octant is (x>cx) + 2(y>cy) + 4(z>cz) against the cell
// centre (src/gravity/octree.h:49-51) and the child centre is the parent
// centre +/- half of the parent half-width (octree.h:56-64).  Level l's digit
// sits in bits [63-3l, 65-3l].
uint64_t octant_key(double px, double py, double pz, const Cube& c, int levels) {
    double x = c.cx, y = c.cy, z = c.cz, h = c.half;
    uint64_t key = 0;
    for (int l = 1; l <= levels; ++l) {
        const int bx = px > x, by = py > y, bz = pz > z;
        const uint64_t oct = static_cast<uint64_t>(bx | (by << 1) | (bz << 2));
        key |= oct << (63 - 3 * l);
        const double hs = h * 0.5;
        x = x + (bx ? hs : -hs);
        y = y + (by ? hs : -hs);
        z = z + (bz ? hs : -hs);
        h = hs;
    }
    return key;
}

struct Params {
    int mode;        // 0 = REF, 1 = ACCURATE
    double theta;
    double eps;
    double G;
    int leaf_cap;
    int quad;
};

struct Tree {
    // Nodes in depth-first pre-order (children in octant order).
    std::vector<int> level, start, count, nchild, leaf;
    std::vector<std::vector<int>> kids;
    std::vector<double> m, cx, cy, cz, half, gx, gy, gz;  // g* = geometric centre
    std::vector<double> q[6];                              // xx yy zz xy xz yz
    std::vector<double> rcrit;
};

struct Sorted {
    std::vector<uint64_t> key;
    std::vector<int64_t> perm;   // sorted position -> original index
    std::vector<double> x, y, z, m;
    std::vector<int> type;
};

Sorted sort_particles(int64_t n, const double* x, const double* y, const double* z,
                      const double* m, const int* type, const Cube& cube) {
    Sorted s;
    std::vector<uint64_t> keys(n);
    for (int64_t i = 0; i < n; ++i) keys[i] = octant_key(x[i], y[i], z[i], cube, kMaxLevel);
    s.perm.resize(n);
    std::iota(s.perm.begin(), s.perm.end(), 0);
    std::stable_sort(s.perm.begin(), s.perm.end(),
                     [&](int64_t a, int64_t b) { return keys[a] < keys[b]; });
    s.key.resize(n); s.x.resize(n); s.y.resize(n); s.z.resize(n); s.m.resize(n); s.type.resize(n);
    for (int64_t p = 0; p < n; ++p) {
        const int64_t i = s.perm[p];
        s.key[p] = keys[i]; s.x[p] = x[i]; s.y[p] = y[i]; s.z[p] = z[i]; s.m[p] = m[i];
        s.type[p] = type ? type[i] : 0;
    }
    return s;
}

inline int digit(uint64_t key, int level) { return static_cast<int>((key >> (63 - 3 * level)) & 7u); }

// A cell with more than leaf_cap bodies is split (the reference splits any
// cell holding two bodies: src/gravity/octree.h:69-87, i.e. leaf_cap = 1);
// cells at the deepest key level stay leaves whatever their count.
int build_node(Tree& t, const Sorted& s, int level, int b, int e, int leaf_cap,
               double gx, double gy, double gz, double half) {
    const int id = static_cast<int>(t.level.size());
    t.level.push_back(level); t.start.push_back(b); t.count.push_back(e - b);
    t.nchild.push_back(0); t.leaf.push_back(1); t.kids.emplace_back();
    t.m.push_back(0); t.cx.push_back(0); t.cy.push_back(0); t.cz.push_back(0);
    t.half.push_back(half); t.gx.push_back(gx); t.gy.push_back(gy); t.gz.push_back(gz);
    for (auto& v : t.q) v.push_back(0);
    t.rcrit.push_back(0);
    if (e - b <= leaf_cap || level >= kMaxLevel) return id;
    t.leaf[id] = 0;
    const double hs = half * 0.5;
    int p = b;
    std::vector<int> kids;
    while (p < e) {
        const int d = digit(s.key[p], level + 1);
        int q = p;
        while (q < e && digit(s.key[q], level + 1) == d) ++q;
        const double cx = gx + ((d & 1) ? hs : -hs);
        const double cy = gy + ((d & 2) ? hs : -hs);
        const double cz = gz + ((d & 4) ? hs : -hs);
        kids.push_back(build_node(t, s, level + 1, p, q, leaf_cap, cx, cy, cz, hs));
        p = q;
    }
    t.kids[id] = kids;
    t.nchild[id] = static_cast<int>(kids.size());
    return id;
}

// Moments with the reference's rules (src/gravity/octree.h:92-127).  A leaf
// holding one body takes that body's mass and position and a zero
// quadrupole.  A leaf holding several bodies (only possible at the deepest
// key level, where the reference would keep subdividing) treats its bodies
// the way an internal node treats one-body children.
void moments_ref(Tree& t, const Sorted& s, int id) {
    if (t.leaf[id] && t.count[id] == 1) {
        const int j = t.start[id];
        t.m[id] = s.m[j]; t.cx[id] = s.x[j]; t.cy[id] = s.y[j]; t.cz[id] = s.z[j];
        return;
    }
    struct Part { double m, x, y, z; };
    std::vector<Part> parts;
    if (t.leaf[id]) {
        for (int j = t.start[id]; j < t.start[id] + t.count[id]; ++j)
            parts.push_back({s.m[j], s.x[j], s.y[j], s.z[j]});
    } else {
        for (int k : t.kids[id]) {
            moments_ref(t, s, k);
            parts.push_back({t.m[k], t.cx[k], t.cy[k], t.cz[k]});
        }
    }
    double m = 0, cx = 0, cy = 0, cz = 0;
    for (const Part& c : parts) {
        if (c.m == 0) continue;
        m += c.m;
        cx += c.x * c.m; cy += c.y * c.m; cz += c.z * c.m;
    }
    if (m > 0) { cx /= m; cy /= m; cz /= m; }
    double qxx = 0, qyy = 0, qzz = 0, qxy = 0, qxz = 0, qyz = 0;
    const double size = t.half[id];
    for (const Part& c : parts) {
        if (c.m == 0) continue;
        const double rx = c.x - cx, ry = c.y - cy, rz = c.z - cz;
        const double r2 = rx * rx + ry * ry + rz * rz + (size * size * 0.01);
        const double mc = c.m;
        qxx += mc * (3.0 * rx * rx - r2);
        qyy += mc * (3.0 * ry * ry - r2);
        qzz += mc * (3.0 * rz * rz - r2);
        qxy += mc * (3.0 * rx * ry);
        qxz += mc * (3.0 * rx * rz);
        qyz += mc * (3.0 * ry * rz);
    }
    t.m[id] = m; t.cx[id] = cx; t.cy[id] = cy; t.cz[id] = cz;
    t.q[0][id] = qxx; t.q[1][id] = qyy; t.q[2][id] = qzz;
    t.q[3][id] = qxy; t.q[4][id] = qxz; t.q[5][id] = qyz;
}

// Moments for the accurate mode: total mass, centre of mass and the traceless
// quadrupole Q = sum m (3 r r^T - r^2 I) about the COM, carried up the tree
// with the parallel-axis terms.  rcrit = 2*half/theta + |COM - centre|.
void moments_accurate(Tree& t, const Sorted& s, int id, double theta) {
    double m = 0, cx = 0, cy = 0, cz = 0;
    double q[6] = {0, 0, 0, 0, 0, 0};
    if (t.leaf[id]) {
        const int b = t.start[id], e = b + t.count[id];
        for (int j = b; j < e; ++j) {
            m += s.m[j];
            cx += s.m[j] * s.x[j]; cy += s.m[j] * s.y[j]; cz += s.m[j] * s.z[j];
        }
        if (m > 0) { cx /= m; cy /= m; cz /= m; } else { cx = t.gx[id]; cy = t.gy[id]; cz = t.gz[id]; }
        for (int j = b; j < e; ++j) {
            const double rx = s.x[j] - cx, ry = s.y[j] - cy, rz = s.z[j] - cz;
            const double r2 = rx * rx + ry * ry + rz * rz;
            const double mj = s.m[j];
            q[0] += mj * (3.0 * rx * rx - r2); q[1] += mj * (3.0 * ry * ry - r2);
            q[2] += mj * (3.0 * rz * rz - r2); q[3] += mj * (3.0 * rx * ry);
            q[4] += mj * (3.0 * rx * rz);      q[5] += mj * (3.0 * ry * rz);
        }
    } else {
        for (int k : t.kids[id]) moments_accurate(t, s, k, theta);
        for (int k : t.kids[id]) {
            m += t.m[k];
            cx += t.m[k] * t.cx[k]; cy += t.m[k] * t.cy[k]; cz += t.m[k] * t.cz[k];
        }
        if (m > 0) { cx /= m; cy /= m; cz /= m; } else { cx = t.gx[id]; cy = t.gy[id]; cz = t.gz[id]; }
        for (int k : t.kids[id]) {
            const double rx = t.cx[k] - cx, ry = t.cy[k] - cy, rz = t.cz[k] - cz;
            const double r2 = rx * rx + ry * ry + rz * rz;
            const double mk = t.m[k];
            q[0] += t.q[0][k] + mk * (3.0 * rx * rx - r2);
            q[1] += t.q[1][k] + mk * (3.0 * ry * ry - r2);
            q[2] += t.q[2][k] + mk * (3.0 * rz * rz - r2);
            q[3] += t.q[3][k] + mk * (3.0 * rx * ry);
            q[4] += t.q[4][k] + mk * (3.0 * rx * rz);
            q[5] += t.q[5][k] + mk * (3.0 * ry * rz);
        }
    }
    t.m[id] = m; t.cx[id] = cx; t.cy[id] = cy; t.cz[id] = cz;
    for (int c = 0; c < 6; ++c) t.q[c][id] = q[c];
    const double ox = cx - t.gx[id], oy = cy - t.gy[id], oz = cz - t.gz[id];
    const double delta = std::sqrt(ox * ox + oy * oy + oz * oz);
    t.rcrit[id] = 2.0 * t.half[id] / theta + delta;
}

// Adaptive softening: src/dt/softening.h:21-35.
inline double next_softening(double size, double mass, double dist) {
    const double eps_size = size * 0.015;
    const double eps_mass = std::cbrt(mass) * 0.002;
    const double taper = 1.0 / (1.0 + dist * 10.0);
    const double eps = (eps_size + eps_mass) * taper;
    return std::max(eps, 1e-4);
}

// One accepted node (or one leaf body) in REF mode: src/gravity/octree.h:138-173.
inline void ref_interact(double nm, double ncx, double ncy, double ncz, double size, const double* Q,
                         double xi, double yi, double zi, double mi, int ti,
                         double& ax, double& ay, double& az) {
    const double dx = ncx - xi, dy = ncy - yi, dz = ncz - zi;
    const double r2 = dx * dx + dy * dy + dz * dz;
    const double dist = std::sqrt(r2 + 1e-20);
    double eps = next_softening(size, nm, dist);
    if (ti == 1) eps = std::max(eps, 2.0 * size / std::pow(nm / mi, 0.333333333));
    const double r2s = r2 + eps * eps;
    const double dinv = 1.0 / std::sqrt(r2s);
    const double inv3 = dinv * dinv * dinv;
    const double fac = 1.0 * nm * inv3;
    ax += dx * fac; ay += dy * fac; az += dz * fac;
    const double inv5 = inv3 * (dinv * dinv);
    const double inv7 = inv5 * (dinv * dinv);
    const double q = Q[0] * dx * dx + Q[1] * dy * dy + Q[2] * dz * dz +
                     2.0 * (Q[3] * dx * dy + Q[4] * dx * dz + Q[5] * dy * dz);
    const double qrx = 2.0 * (Q[0] * dx + Q[3] * dy + Q[4] * dz);
    const double qry = 2.0 * (Q[3] * dx + Q[1] * dy + Q[5] * dz);
    const double qrz = 2.0 * (Q[4] * dx + Q[5] * dy + Q[2] * dz);
    ax += 0.5 * (qrx * inv5 - 5.0 * q * inv7 * dx);
    ay += 0.5 * (qry * inv5 - 5.0 * q * inv7 * dy);
    az += 0.5 * (qrz * inv5 - 5.0 * q * inv7 * dz);
}

// bhAccel (src/gravity/octree.h:133-179) for the body at sorted position i.
void walk_ref(const Tree& t, const Sorted& s, int id, int i, double theta,
              double& ax, double& ay, double& az) {
    if (t.m[id] == 0) return;
    const bool leaf = t.leaf[id];
    if (leaf && t.count[id] == 1 && t.start[id] == i) return;
    const double Q[6] = {t.q[0][id], t.q[1][id], t.q[2][id], t.q[3][id], t.q[4][id], t.q[5][id]};
    if (leaf && t.count[id] > 1) {
        // Deepest-level bucket: its bodies act as one-body leaves of this size.
        static const double Z[6] = {0, 0, 0, 0, 0, 0};
        for (int j = t.start[id]; j < t.start[id] + t.count[id]; ++j) {
            if (j == i || s.m[j] == 0) continue;
            ref_interact(s.m[j], s.x[j], s.y[j], s.z[j], t.half[id], Z,
                         s.x[i], s.y[i], s.z[i], s.m[i], s.type[i], ax, ay, az);
        }
        return;
    }
    const double dx = t.cx[id] - s.x[i], dy = t.cy[id] - s.y[i], dz = t.cz[id] - s.z[i];
    const double r2 = dx * dx + dy * dy + dz * dz;
    const double dist = std::sqrt(r2 + 1e-20);
    if (leaf || (t.half[id] / dist) < theta) {
        ref_interact(t.m[id], t.cx[id], t.cy[id], t.cz[id], t.half[id], Q,
                     s.x[i], s.y[i], s.z[i], s.m[i], s.type[i], ax, ay, az);
        return;
    }
    for (int k : t.kids[id]) walk_ref(t, s, k, i, theta, ax, ay, az);
}

struct Acc { double ax = 0, ay = 0, az = 0, pot = 0; int64_t npp = 0, npc = 0; };

// Accurate-mode walk for the body at sorted position i: a node is used as a
// multipole when |COM - x_i| >= rcrit; an opened leaf is summed body by body.
void walk_accurate(const Tree& t, const Sorted& s, const Params& P, int id, int i, Acc& a) {
    if (t.m[id] == 0) return;
    const double dx = t.cx[id] - s.x[i], dy = t.cy[id] - s.y[i], dz = t.cz[id] - s.z[i];
    const double r2 = dx * dx + dy * dy + dz * dz;
    const double eps2 = P.eps * P.eps;
    if (r2 < t.rcrit[id] * t.rcrit[id]) {
        if (!t.leaf[id]) {
            for (int k : t.kids[id]) walk_accurate(t, s, P, k, i, a);
            return;
        }
        for (int j = t.start[id]; j < t.start[id] + t.count[id]; ++j) {
            if (j == i) continue;
            const double ex = s.x[j] - s.x[i], ey = s.y[j] - s.y[i], ez = s.z[j] - s.z[i];
            const double e2 = ex * ex + ey * ey + ez * ez + eps2;
            const double rinv = 1.0 / std::sqrt(e2);
            const double mr3 = P.G * s.m[j] * rinv * rinv * rinv;
            a.ax += mr3 * ex; a.ay += mr3 * ey; a.az += mr3 * ez;
            a.pot -= P.G * s.m[j] * rinv;
            ++a.npp;
        }
        return;
    }
    const double r2s = r2 + eps2;
    const double rinv = 1.0 / std::sqrt(r2s);
    const double rinv2 = rinv * rinv;
    const double mr3 = P.G * t.m[id] * rinv * rinv2;
    a.ax += mr3 * dx; a.ay += mr3 * dy; a.az += mr3 * dz;
    a.pot -= P.G * t.m[id] * rinv;
    if (P.quad) {
        const double qxx = t.q[0][id], qyy = t.q[1][id], qzz = t.q[2][id];
        const double qxy = t.q[3][id], qxz = t.q[4][id], qyz = t.q[5][id];
        const double qdx = qxx * dx + qxy * dy + qxz * dz;
        const double qdy = qxy * dx + qyy * dy + qyz * dz;
        const double qdz = qxz * dx + qyz * dy + qzz * dz;
        const double q = dx * qdx + dy * qdy + dz * qdz;
        const double rinv5 = rinv2 * rinv2 * rinv;
        const double rinv7 = rinv5 * rinv2;
        const double c7 = 2.5 * P.G * q * rinv7;
        const double c5 = P.G * rinv5;
        a.ax += c7 * dx - c5 * qdx;
        a.ay += c7 * dy - c5 * qdy;
        a.az += c7 * dz - c5 * qdz;
        a.pot -= 0.5 * P.G * q * rinv5;
    }
    ++a.npc;
}

Tree build_tree(const Sorted& s, const Cube& cube, int leaf_cap) {
    Tree t;
    const int n = static_cast<int>(s.key.size());
    build_node(t, s, 0, 0, n, leaf_cap, cube.cx, cube.cy, cube.cz, cube.half);
    return t;
}

void accel_all(int64_t n, const double* x, const double* y, const double* z,
               const double* m, const int* type, const Params& P,
               double* ax, double* ay, double* az, double* pot, int64_t* counts) {
    if (n <= 0) return;
    const Cube cube = root_cube(n, x, y, z);
    Sorted s = sort_particles(n, x, y, z, m, type, cube);
    Tree t = build_tree(s, cube, P.mode == 0 ? 1 : P.leaf_cap);
    if (P.mode == 0) moments_ref(t, s, 0);
    else moments_accurate(t, s, 0, P.theta);
    int64_t npp = 0, npc = 0;
    #pragma omp parallel for schedule(dynamic, 64) reduction(+ : npp, npc)
    for (int64_t p = 0; p < n; ++p) {
        const int64_t i = s.perm[p];
        if (P.mode == 0) {
            double a0 = 0, a1 = 0, a2 = 0;
            walk_ref(t, s, 0, static_cast<int>(p), P.theta, a0, a1, a2);
            ax[i] = a0; ay[i] = a1; az[i] = a2;
            if (pot) pot[i] = 0;
        } else {
            Acc a;
            walk_accurate(t, s, P, 0, static_cast<int>(p), a);
            ax[i] = a.ax; ay[i] = a.ay; az[i] = a.az;
            if (pot) pot[i] = a.pot;
            npp += a.npp; npc += a.npc;
        }
    }
    if (counts) { counts[0] = npp; counts[1] = npc; counts[2] = static_cast<int64_t>(t.level.size()); }
}

}  // namespace

extern "C" {

void orc_root_cube(int64_t n, const double* x, const double* y, const double* z, double* out4) {
    const Cube c = root_cube(n, x, y, z);
    out4[0] = c.cx; out4[1] = c.cy; out4[2] = c.cz; out4[3] = c.half;
}

// Keys against a given root cube (cube4 = cx, cy, cz, half).
void orc_keys(int64_t n, const double* x, const double* y, const double* z,
              const double* cube4, int levels, uint64_t* keys) {
    const Cube c{cube4[0], cube4[1], cube4[2], cube4[3]};
    for (int64_t i = 0; i < n; ++i) keys[i] = octant_key(x[i], y[i], z[i], c, levels);
}

// Stable key order: perm[p] is the original index of the p-th smallest key.
void orc_sort(int64_t n, const uint64_t* keys, int64_t* perm) {
    std::vector<int64_t> p(n);
    std::iota(p.begin(), p.end(), 0);
    std::stable_sort(p.begin(), p.end(), [&](int64_t a, int64_t b) { return keys[a] < keys[b]; });
    std::memcpy(perm, p.data(), sizeof(int64_t) * n);
}

// mode 0 = REF, 1 = ACCURATE.  counts (optional) = {PP, PC, nodes}.
int orc_accel(int64_t n, const double* x, const double* y, const double* z,
              const double* m, const int* type, int mode, double theta, double eps,
              double G, int leaf_cap, int quad,
              double* ax, double* ay, double* az, double* pot, int64_t* counts) {
    Params P{mode, theta, eps, G, leaf_cap < 1 ? 1 : leaf_cap, quad};
    accel_all(n, x, y, z, m, type, P, ax, ay, az, pot, counts);
    return 0;
}

// FP64 direct summation with Plummer softening for the k bodies listed in idx.
int orc_direct(int64_t n, const double* x, const double* y, const double* z, const double* m,
               double eps, double G, int64_t k, const int64_t* idx,
               double* ax, double* ay, double* az, double* pot) {
    const double eps2 = eps * eps;
    #pragma omp parallel for schedule(dynamic, 4)
    for (int64_t t = 0; t < k; ++t) {
        const int64_t i = idx[t];
        double a0 = 0, a1 = 0, a2 = 0, ph = 0;
        for (int64_t j = 0; j < n; ++j) {
            if (j == i) continue;
            const double dx = x[j] - x[i], dy = y[j] - y[i], dz = z[j] - z[i];
            const double r2 = dx * dx + dy * dy + dz * dz + eps2;
            const double rinv = 1.0 / std::sqrt(r2);
            const double mr3 = G * m[j] * rinv * rinv * rinv;
            a0 += mr3 * dx; a1 += mr3 * dy; a2 += mr3 * dz;
            ph -= G * m[j] * rinv;
        }
        ax[t] = a0; ay[t] = a1; az[t] = a2;
        if (pot) pot[t] = ph;
    }
    return 0;
}

// KDK leapfrog with the structure of src/gravity/step.h:111-189: forces at
// x_n, v += a dt/2, x += v dt, forces at x_{n+1}, v += a dt/2.
int orc_step(int64_t n, double* x, double* y, double* z, double* vx, double* vy, double* vz,
             const double* m, const int* type, int mode, double theta, double eps, double G,
             int leaf_cap, int quad, double dt, int nsteps) {
    Params P{mode, theta, eps, G, leaf_cap < 1 ? 1 : leaf_cap, quad};
    std::vector<double> ax(n), ay(n), az(n);
    const double half = dt * 0.5;
    for (int s = 0; s < nsteps; ++s) {
        accel_all(n, x, y, z, m, type, P, ax.data(), ay.data(), az.data(), nullptr, nullptr);
        for (int64_t i = 0; i < n; ++i) { vx[i] += ax[i] * half; vy[i] += ay[i] * half; vz[i] += az[i] * half; }
        for (int64_t i = 0; i < n; ++i) { x[i] += vx[i] * dt; y[i] += vy[i] * dt; z[i] += vz[i] * dt; }
        accel_all(n, x, y, z, m, type, P, ax.data(), ay.data(), az.data(), nullptr, nullptr);
        for (int64_t i = 0; i < n; ++i) { vx[i] += ax[i] * half; vy[i] += ay[i] * half; vz[i] += az[i] * half; }
    }
    return 0;
}

// Adaptive step: src/dt/adaptive.h:23-52.
double orc_adaptive_dt(int64_t n, const double* vx, const double* vy, const double* vz, double base_dt) {
    double vmax2 = 0;
    for (int64_t i = 0; i < n; ++i) {
        const double s2 = vx[i] * vx[i] + vy[i] * vy[i] + vz[i] * vz[i];
        if (s2 > vmax2) vmax2 = s2;
    }
    double v = std::sqrt(vmax2);
    v = std::min(v, 1e4);
    if (v < 1e-8) return base_dt;
    double dt = base_dt / (1 + v);
    dt = std::max(dt, base_dt * 0.01);
    dt = std::min(dt, base_dt * 1.0);
    return dt;
}

// Depth-first tree export in the row format of ref_tree_export (16 doubles
// per node; body_index = original index of a one-body leaf, else -1).
// mode selects the moment rules.  Returns the node count.
int64_t orc_tree_export(int64_t n, const double* x, const double* y, const double* z,
                        const double* m, int mode, double theta, int leaf_cap,
                        double* rows, int64_t cap) {
    if (n <= 0) return 0;
    const Cube cube = root_cube(n, x, y, z);
    Sorted s = sort_particles(n, x, y, z, m, nullptr, cube);
    Tree t = build_tree(s, cube, mode == 0 ? 1 : (leaf_cap < 1 ? 1 : leaf_cap));
    if (mode == 0) moments_ref(t, s, 0); else moments_accurate(t, s, 0, theta);
    const int64_t nn = static_cast<int64_t>(t.level.size());
    for (int64_t id = 0; id < nn && id < cap; ++id) {
        double* r = rows + 16 * id;
        r[0] = t.level[id]; r[1] = t.m[id]; r[2] = t.cx[id]; r[3] = t.cy[id]; r[4] = t.cz[id];
        r[5] = t.half[id];
        for (int c = 0; c < 6; ++c) r[6 + c] = t.q[c][id];
        r[12] = t.leaf[id];
        r[13] = (t.leaf[id] && t.count[id] == 1) ? static_cast<double>(s.perm[t.start[id]]) : -1.0;
        r[14] = t.gx[id];
        r[15] = t.count[id];
    }
    return nn;
}

}  // extern "C"
