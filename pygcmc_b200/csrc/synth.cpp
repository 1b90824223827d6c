// Synthetic fixed-atom generators for the benchmark systems (host code).
//
// A confined self-avoiding random-walk chain: fixed-length steps in uniformly
// random directions, kept inside a sphere (or a slab with an optional
// cylindrical pore) and away from every non-bonded atom placed so far
// (bonded = the two preceding atoms).  When a step cannot be placed after a
// bounded number of trials the chain restarts at a random free point (a chain
// break).  A cell hash of side `excl` makes each trial O(1).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <unordered_map>
#include <vector>

namespace {

struct SplitMix64 {
    uint64_t s;
    explicit SplitMix64(uint64_t seed) : s(seed) {}
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};

struct Region {
    int kind;          // 0 sphere, 1 slab
    double c[3];       // sphere centre / slab: pore axis (x,y) and slab centre z
    double radius;     // sphere radius
    double half;       // slab half thickness (z)
    double lo[2], hi[2];  // slab lateral extent (x, y)
    double pore;       // slab: pore radius around (c[0], c[1]); 0 = none
    bool inside(const double p[3]) const {
        if (kind == 0) {
            double dx = p[0] - c[0], dy = p[1] - c[1], dz = p[2] - c[2];
            return dx * dx + dy * dy + dz * dz <= radius * radius;
        }
        if (std::fabs(p[2] - c[2]) > half) return false;
        if (p[0] < lo[0] || p[0] >= hi[0] || p[1] < lo[1] || p[1] >= hi[1]) return false;
        double dx = p[0] - c[0], dy = p[1] - c[1];
        return dx * dx + dy * dy >= pore * pore;
    }
    void random_point(SplitMix64& r, double p[3]) const {
        for (;;) {
            if (kind == 0) {
                for (int i = 0; i < 3; ++i) p[i] = c[i] + (2.0 * r.uniform() - 1.0) * radius;
            } else {
                p[0] = lo[0] + r.uniform() * (hi[0] - lo[0]);
                p[1] = lo[1] + r.uniform() * (hi[1] - lo[1]);
                p[2] = c[2] + (2.0 * r.uniform() - 1.0) * half;
            }
            if (inside(p)) return;
        }
    }
};

struct CellHash {
    double h;
    std::unordered_map<int64_t, std::vector<int>> cells;
    explicit CellHash(double side) : h(side) {}
    static int64_t key(int64_t x, int64_t y, int64_t z) {
        return ((x + 1048576) << 42) ^ ((y + 1048576) << 21) ^ (z + 1048576);
    }
    void add(const double p[3], int id) {
        cells[key((int64_t)std::floor(p[0] / h), (int64_t)std::floor(p[1] / h),
                  (int64_t)std::floor(p[2] / h))].push_back(id);
    }
    // true when no atom other than the excluded ids lies within h of p
    bool clear(const double p[3], const std::vector<double>& xyz, int skip_from, int skip_to) const {
        int64_t cx = (int64_t)std::floor(p[0] / h), cy = (int64_t)std::floor(p[1] / h),
                cz = (int64_t)std::floor(p[2] / h);
        double h2 = h * h;
        for (int64_t dx = -1; dx <= 1; ++dx)
            for (int64_t dy = -1; dy <= 1; ++dy)
                for (int64_t dz = -1; dz <= 1; ++dz) {
                    auto it = cells.find(key(cx + dx, cy + dy, cz + dz));
                    if (it == cells.end()) continue;
                    for (int j : it->second) {
                        if (j >= skip_from && j <= skip_to) continue;
                        double ex = xyz[3 * j] - p[0], ey = xyz[3 * j + 1] - p[1], ez = xyz[3 * j + 2] - p[2];
                        if (ex * ex + ey * ey + ez * ez < h2) return false;
                    }
                }
        return true;
    }
};

int grow_chain(const Region& reg, int n, double step, double excl, uint64_t seed, float* out, int* n_breaks) {
    SplitMix64 r(seed);
    std::vector<double> xyz((size_t)n * 3);
    CellHash hash(excl);
    int breaks = 0;
    double p[3];
    for (int i = 0; i < n; ++i) {
        bool placed = false;
        if (i > 0) {
            for (int t = 0; t < 64 && !placed; ++t) {
                double z = 2.0 * r.uniform() - 1.0, phi = 2.0 * M_PI * r.uniform();
                double s = std::sqrt(std::max(0.0, 1.0 - z * z));
                p[0] = xyz[3 * (i - 1)] + step * s * std::cos(phi);
                p[1] = xyz[3 * (i - 1) + 1] + step * s * std::sin(phi);
                p[2] = xyz[3 * (i - 1) + 2] + step * z;
                if (!reg.inside(p)) continue;
                placed = hash.clear(p, xyz, i - 2, i - 1);
            }
        }
        if (!placed) {
            if (i > 0) ++breaks;
            int t = 0;
            for (; t < 200000; ++t) {
                reg.random_point(r, p);
                if (hash.clear(p, xyz, -1, -1)) break;
            }
            if (t == 200000) return -1;  // region full
        }
        for (int k = 0; k < 3; ++k) xyz[3 * i + k] = p[k];
        hash.add(p, i);
    }
    for (size_t k = 0; k < xyz.size(); ++k) out[k] = (float)xyz[k];
    if (n_breaks) *n_breaks = breaks;
    return 0;
}

// Periodic cell hash over a box (for rigid-body placement).
struct PeriodicHash {
    double lo[3], L[3], h;
    int n[3];
    std::vector<std::vector<double>> cells;  // xyz triples per cell
    PeriodicHash(const double lo_[3], const double L_[3], double side) : h(side) {
        for (int i = 0; i < 3; ++i) {
            lo[i] = lo_[i];
            L[i] = L_[i];
            n[i] = std::max(1, (int)std::floor(L[i] / side));
        }
        cells.resize((size_t)n[0] * n[1] * n[2]);
    }
    int idx(int a, int i) const { return ((a % n[i]) + n[i]) % n[i]; }
    int coord(double x, int i) const { return idx((int)std::floor((x - lo[i]) / L[i] * n[i]), i); }
    void add(const double p[3]) {
        auto& c = cells[((size_t)coord(p[2], 2) * n[1] + coord(p[1], 1)) * n[0] + coord(p[0], 0)];
        c.insert(c.end(), p, p + 3);
    }
    bool clear(const double p[3], double r) const {
        const int cx = coord(p[0], 0), cy = coord(p[1], 1), cz = coord(p[2], 2);
        const int rx = std::min(n[0], 3), ry = std::min(n[1], 3), rz = std::min(n[2], 3);
        for (int dz = 0; dz < rz; ++dz)
            for (int dy = 0; dy < ry; ++dy)
                for (int dx = 0; dx < rx; ++dx) {
                    const auto& c = cells[((size_t)idx(cz + dz - (rz > 1), 2) * n[1] + idx(cy + dy - (ry > 1), 1)) * n[0] +
                                          idx(cx + dx - (rx > 1), 0)];
                    for (size_t k = 0; k < c.size(); k += 3) {
                        double d2 = 0.0;
                        for (int i = 0; i < 3; ++i) {
                            double d = c[k + i] - p[i];
                            d -= L[i] * std::round(d / L[i]);
                            d2 += d * d;
                        }
                        if (d2 < r * r) return false;
                    }
                }
        return true;
    }
};

}  // namespace

extern "C" {

// `count` copies of a rigid template (nsites x 3, centred) at uniformly random
// positions and orientations in the periodic box [lo, lo+L), each site at
// least min_dist from every atom already present (existing atoms and earlier
// copies).  Returns 0, or -1 when a copy cannot be placed.
int gcmc_synth_place(int n_existing, const float* existing_xyz, const float lo[3], const float L[3],
                     const float* tpl_xyz, int nsites, int count, float min_dist, uint64_t seed,
                     float* out_xyz) {
    double lo_d[3] = {lo[0], lo[1], lo[2]}, L_d[3] = {L[0], L[1], L[2]};
    PeriodicHash hash(lo_d, L_d, std::max(1e-3, (double)min_dist));
    for (int a = 0; a < n_existing; ++a) {
        double p[3] = {existing_xyz[3 * a], existing_xyz[3 * a + 1], existing_xyz[3 * a + 2]};
        hash.add(p);
    }
    SplitMix64 r(seed);
    std::vector<double> site((size_t)nsites * 3);
    for (int c = 0; c < count; ++c) {
        bool placed = false;
        for (int t = 0; t < 200000 && !placed; ++t) {
            // uniform rotation (Shoemake) and uniform position
            const double u1 = r.uniform(), u2 = 2 * M_PI * r.uniform(), u3 = 2 * M_PI * r.uniform();
            const double a = std::sqrt(1 - u1), b = std::sqrt(u1);
            const double x = a * std::sin(u2), y = a * std::cos(u2), z = b * std::sin(u3), w = b * std::cos(u3);
            const double R[3][3] = {{1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)},
                                    {2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)},
                                    {2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)}};
            double cen[3];
            for (int i = 0; i < 3; ++i) cen[i] = lo_d[i] + r.uniform() * L_d[i];
            placed = true;
            for (int s = 0; s < nsites && placed; ++s) {
                for (int i = 0; i < 3; ++i)
                    site[3 * s + i] = cen[i] + R[i][0] * tpl_xyz[3 * s] + R[i][1] * tpl_xyz[3 * s + 1] +
                                      R[i][2] * tpl_xyz[3 * s + 2];
                placed = hash.clear(&site[3 * s], min_dist);
            }
        }
        if (!placed) return -1;
        for (int s = 0; s < nsites; ++s) {
            hash.add(&site[3 * s]);
            for (int i = 0; i < 3; ++i) out_xyz[((size_t)c * nsites + s) * 3 + i] = (float)site[3 * s + i];
        }
    }
    return 0;
}


// Chain of n atoms inside a sphere; returns 0, or -1 when the sphere cannot hold it.
int gcmc_synth_chain_sphere(int n, const float centre[3], float radius, float step, float excl,
                            uint64_t seed, float* out_xyz, int* n_breaks) {
    Region reg{};
    reg.kind = 0;
    for (int i = 0; i < 3; ++i) reg.c[i] = centre[i];
    reg.radius = radius;
    return grow_chain(reg, n, step, excl, seed, out_xyz, n_breaks);
}

// Chain of n atoms inside the slab |z - zc| <= half, x in [lo0,hi0), y in [lo1,hi1),
// outside a cylinder of radius `pore` along z through (px, py).
int gcmc_synth_chain_slab(int n, float lo0, float hi0, float lo1, float hi1, float zc, float half,
                          float px, float py, float pore, float step, float excl, uint64_t seed,
                          float* out_xyz, int* n_breaks) {
    Region reg{};
    reg.kind = 1;
    reg.c[0] = px; reg.c[1] = py; reg.c[2] = zc;
    reg.half = half;
    reg.lo[0] = lo0; reg.hi[0] = hi0; reg.lo[1] = lo1; reg.hi[1] = hi1;
    reg.pore = pore;
    return grow_chain(reg, n, step, excl, seed, out_xyz, n_breaks);
}

}  // extern "C"
