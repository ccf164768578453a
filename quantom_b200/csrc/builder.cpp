// Box assembly helpers (host C++): the B200 build's counterpart of the
// reference's solvent placement (BoxBuilder::solvateBox/spaceAvailable,
// Quantom/Quantom/BoxBuilder.cu:194-218, 440-461).  The reference rejects a
// candidate solvent closer than a minimum distance to anything already placed.
// Near the packing fractions of the benchmark boxes (phi ~ 0.377 at
// 0.28 nm) sequential rejection approaches the random-sequential-addition
// jamming limit and needs ~1e9 trials, so this builder samples the same target
// — positions uniform in the box conditioned on no pair closer than d_min —
// with a hard-sphere Monte Carlo chain started from a lattice:
//   1. an FCC lattice whose nearest-neighbour distance is >= d_min; sites
//      closer than d_min to a fixed particle (chain beads) are dropped and the
//      requested number of sites is drawn at random;
//   2. n_sweeps Metropolis sweeps of uniform trial displacements, rejected on
//      any overlap (cell list, minimum image), step size tuned toward ~40%
//      acceptance.
// Deterministic for a given seed (xoshiro256** seeded by splitmix64).
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>

namespace {

struct Rng {
    uint64_t s[4];
    static uint64_t splitmix(uint64_t& x) {
        uint64_t z = (x += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    explicit Rng(uint64_t seed) {
        for (auto& v : s) v = splitmix(seed);
    }
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next() {
        const uint64_t r = rotl(s[1] * 5, 7) * 9;
        const uint64_t t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return r;
    }
    double uniform() { return static_cast<double>(next() >> 11) * (1.0 / 9007199254740992.0); }
    uint64_t below(uint64_t n) { return static_cast<uint64_t>(uniform() * static_cast<double>(n)) % n; }
};

inline double wrap(double x, double L) {
    x = std::fmod(x, L);
    return x < 0 ? x + L : x;
}

struct CellGrid {
    int m = 1;
    double L = 1, cell = 1;
    std::vector<std::vector<int>> cells;
    void init(double box, double min_cell) {
        L = box;
        m = std::max(1, static_cast<int>(std::floor(box / min_cell)));
        cell = box / m;
        cells.assign(static_cast<size_t>(m) * m * m, {});
    }
    int index(const double* p) const {
        int ix = std::min(m - 1, static_cast<int>(p[0] / cell));
        int iy = std::min(m - 1, static_cast<int>(p[1] / cell));
        int iz = std::min(m - 1, static_cast<int>(p[2] / cell));
        return (ix * m + iy) * m + iz;
    }
    void insert(int id, const double* p) { cells[index(p)].push_back(id); }
    void remove(int id, const double* p) {
        auto& v = cells[index(p)];
        auto it = std::find(v.begin(), v.end(), id);
        if (it != v.end()) {
            *it = v.back();
            v.pop_back();
        }
    }
};

// True if p is at least d_min from every particle in the grid other than
// `self` (and at least fixed_rmin[id] from fixed particle id, if given).
bool is_free(const CellGrid& g, const std::vector<double>& pos, const double* p, int self, double d2min,
             const double* fixed_rmin = nullptr, int n_fixed = 0) {
    const int m = g.m;
    const int cx = std::min(m - 1, static_cast<int>(p[0] / g.cell));
    const int cy = std::min(m - 1, static_cast<int>(p[1] / g.cell));
    const int cz = std::min(m - 1, static_cast<int>(p[2] / g.cell));
    const int span = m >= 3 ? 1 : 0;
    for (int dx = -span; dx <= span; dx++)
        for (int dy = -span; dy <= span; dy++)
            for (int dz = -span; dz <= span; dz++) {
                const int ix = (cx + dx + m) % m, iy = (cy + dy + m) % m, iz = (cz + dz + m) % m;
                for (int id : g.cells[(ix * m + iy) * m + iz]) {
                    if (id == self) continue;
                    double d2 = 0;
                    for (int k = 0; k < 3; k++) {
                        double d = pos[3 * id + k] - p[k];
                        d -= g.L * std::nearbyint(d / g.L);
                        d2 += d * d;
                    }
                    const double lim = (fixed_rmin && id < n_fixed) ? fixed_rmin[id] * fixed_rmin[id] : d2min;
                    if (d2 < lim) return false;
                }
            }
    if (m < 3) {  // tiny boxes: fall back to all particles
        for (size_t id = 0; id < pos.size() / 3; id++) {
            if (static_cast<int>(id) == self) continue;
            double d2 = 0;
            for (int k = 0; k < 3; k++) {
                double d = pos[3 * id + k] - p[k];
                d -= g.L * std::nearbyint(d / g.L);
                d2 += d * d;
            }
            const double lim = (fixed_rmin && static_cast<int>(id) < n_fixed) ? fixed_rmin[id] * fixed_rmin[id] : d2min;
            if (d2 < lim) return false;
        }
    }
    return true;
}

}  // namespace

extern "C" {

// Places n_mobile points in the periodic cube [0, box)^3, none closer than
// d_min to each other, nor closer than fixed_rmin[k] (or d_min when
// fixed_rmin is NULL) to fixed point k of `fixed_xyz` (which must lie in the
// box).  Writes n_mobile*3 doubles to out_xyz.  Returns the number of accepted
// Monte Carlo moves (>= 0), or -1 if the lattice cannot hold n_mobile points.
long lima_builder_pack_spheres(double box, double d_min, const double* fixed_xyz, const double* fixed_rmin,
                               int n_fixed, int n_mobile, unsigned long long seed, int n_sweeps, double* out_xyz) {
    Rng rng(seed);
    const double d2min = d_min * d_min;
    const int n_tot = n_fixed + n_mobile;
    double cell_min = d_min;
    for (int i = 0; fixed_rmin && i < n_fixed; i++) cell_min = std::max(cell_min, fixed_rmin[i]);
    std::vector<double> pos(static_cast<size_t>(n_tot) * 3);
    for (int i = 0; i < 3 * n_fixed; i++) pos[i] = wrap(fixed_xyz[i], box);
    CellGrid fixed_grid;
    fixed_grid.init(box, cell_min);
    for (int i = 0; i < n_fixed; i++) fixed_grid.insert(i, &pos[3 * i]);

    // 1. lattice sites
    std::vector<double> sites;
    for (int M = std::max(1, static_cast<int>(std::cbrt(n_mobile / 4.0))); ; M++) {
        const double a = box / M;
        if (a / std::sqrt(2.0) < d_min) return -1;
        sites.clear();
        static const double basis[4][3] = {{0, 0, 0}, {0.5, 0.5, 0}, {0.5, 0, 0.5}, {0, 0.5, 0.5}};
        for (int i = 0; i < M; i++)
            for (int j = 0; j < M; j++)
                for (int k = 0; k < M; k++)
                    for (auto& b : basis) {
                        double p[3] = {(i + b[0] + 0.25) * a, (j + b[1] + 0.25) * a, (k + b[2] + 0.25) * a};
                        if (n_fixed == 0 || is_free(fixed_grid, pos, p, -1, d2min, fixed_rmin, n_fixed))
                            sites.insert(sites.end(), p, p + 3);
                    }
        if (static_cast<int>(sites.size() / 3) >= n_mobile) break;
    }
    // random subset (partial Fisher-Yates)
    const size_t n_sites = sites.size() / 3;
    std::vector<size_t> order(n_sites);
    for (size_t i = 0; i < n_sites; i++) order[i] = i;
    for (int i = 0; i < n_mobile; i++) {
        size_t j = i + rng.below(n_sites - i);
        std::swap(order[i], order[j]);
    }
    CellGrid grid;
    grid.init(box, cell_min);
    for (int i = 0; i < n_fixed; i++) grid.insert(i, &pos[3 * i]);
    for (int i = 0; i < n_mobile; i++) {
        double* p = &pos[3 * (n_fixed + i)];
        std::memcpy(p, &sites[3 * order[i]], 3 * sizeof(double));
        grid.insert(n_fixed + i, p);
    }

    // 2. hard-sphere Metropolis sweeps
    double step = 0.25 * d_min;
    long accepted_total = 0;
    for (int sweep = 0; sweep < n_sweeps; sweep++) {
        long acc = 0;
        for (int t = 0; t < n_mobile; t++) {
            const int id = n_fixed + static_cast<int>(rng.below(n_mobile));
            double* p = &pos[3 * id];
            double trial[3];
            for (int k = 0; k < 3; k++) trial[k] = wrap(p[k] + (2.0 * rng.uniform() - 1.0) * step, box);
            if (is_free(grid, pos, trial, id, d2min, fixed_rmin, n_fixed)) {
                grid.remove(id, p);
                std::memcpy(p, trial, sizeof(trial));
                grid.insert(id, p);
                acc++;
            }
        }
        accepted_total += acc;
        const double rate = n_mobile ? static_cast<double>(acc) / n_mobile : 0.4;
        step *= (rate > 0.4) ? 1.1 : 0.9;
        step = std::min(std::max(step, 0.01 * d_min), 0.5 * box);
    }
    std::memcpy(out_xyz, &pos[3 * n_fixed], sizeof(double) * 3 * n_mobile);
    return accepted_total;
}

}  // extern "C"
